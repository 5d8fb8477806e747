/*
 * qa_oracle.c -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * A plain-C, single-threaded restatement of qanneal's Monte Carlo sweep
 * engine, written so that its results can be compared bit for bit with the
 * CUDA engine in qlatanneal_b200/csrc.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg may load it.
 *
 * What it restates (file:line in the qanneal sources):
 *   DenseIsing       src/dense_ising.cpp:29-106   (energy, local fields, flip update)
 *   SparseIsing      src/sparse_ising.cpp:35-102
 *   HigherOrderIsing src/higher_order_ising.cpp:10-206 (term consolidation, energy,
 *                    fields, update after flip)
 *   SA               src/annealer.cpp:33-75
 *   SQA run()        src/sqa_annealer.cpp:87-477 (slice + worldline sweeps,
 *                    per-step energy scan and best tracking)
 *   SQA-PT run()     src/sqa_parallel_tempering.cpp:81-346
 *   SQA-Chi run_chi  src/sqa_chi_annealer.cpp:81-438
 *   cluster moves    src/sqa_annealer.cpp:215-288, src/sqa_parallel_tempering.cpp:222-278
 *   classical PT     src/parallel_tempering.cpp:36-122 (the SQA-PT core, one slice)
 *   replicas         src/replica_annealer.cpp:46-142 (SA reads + magnetisation)
 *   SQA run_optimal  src/sqa_annealer.cpp:499-952 (beta ramp, chi_B calibration, J_perp trajectory)
 *   SQA-PT run_optimal src/sqa_parallel_tempering.cpp:348-882
 *
 * The "replay model".  The qanneal loops draw from std::mt19937_64 through
 * libstdc++ distributions and visit spins in std::shuffle order, which no GPU
 * can reproduce.  Both this file and the CUDA engine therefore follow one
 * shared definition of the random stream, the visit order and the float32
 * acceptance rule, and are required to agree exactly:
 *   - Philox4x32-10 counter RNG (Salmon et al., SC'11), key = seed + read,
 *     counter = (spin slot, cell, sweep, domain tag).
 *   - Trotter slices are swept in phases of equal parity (even, odd, and the
 *     last slice alone when P is odd), spins in ascending order inside a slice.
 *   - Local fields g = J.s (h kept apart) in float32, couplings rounded to
 *     float32, field init accumulated in float64 then rounded.
 *   - Metropolis test on y = -dE in float32: y = x*B - trotter with
 *     x = s*(h+g), B = 2*beta/P (2*beta for SA), trotter = 2 J_perp s (s_prev +
 *     s_next); accept iff y >= 0 or (y > -17 and u < e^y), with a
 *     deterministic float32 e^y (Taylor series of 2^f) computed identically
 *     on both sides.
 *   - Energies for the per-step scan in float64, summed in "warp order"
 *     (32 lane-strided partial sums, then an xor butterfly):
 *     E = c + (sum s h + sum s g / 2) for quadratic models.
 * For integer couplings every value is exact, so spins, accept decisions,
 * energies and traces agree bit for bit.  Parity with the unmodified qanneal
 * code is checked separately (statistically, and exactly on the golden
 * energy/field vectors) against the reference compiled under oracle/_ref.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_EXPORT __attribute__((visibility("default")))

/* ------------------------------------------------------------------ */
/* Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel random numbers: */
/* as easy as 1, 2, 3", SC'11).                                          */
/* ------------------------------------------------------------------ */
#define PH_M0 0xD2511F53u
#define PH_M1 0xCD9E8D57u
#define PH_W0 0x9E3779B9u
#define PH_W1 0xBB67AE85u

OR_EXPORT void or_philox(const uint32_t ctr_in[4], const uint32_t key_in[2], uint32_t out[4]) {
    uint32_t c0 = ctr_in[0], c1 = ctr_in[1], c2 = ctr_in[2], c3 = ctr_in[3];
    uint32_t k0 = key_in[0], k1 = key_in[1];
    for (int r = 0; r < 10; ++r) {
        uint64_t p0 = (uint64_t)PH_M0 * (uint64_t)c0;
        uint64_t p1 = (uint64_t)PH_M1 * (uint64_t)c2;
        uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
        uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
        uint32_t n0 = hi1 ^ c1 ^ k0;
        uint32_t n2 = hi0 ^ c3 ^ k1;
        c0 = n0; c1 = lo1; c2 = n2; c3 = lo0;
        k0 += PH_W0; k1 += PH_W1;
    }
    out[0] = c0; out[1] = c1; out[2] = c2; out[3] = c3;
}

/* Domain tags (counter word 3, low byte). */
enum {
    DOM_INIT = 1, DOM_SA = 2, DOM_SLICE = 3, DOM_WORLD = 4, DOM_SWAP = 5,
    DOM_PILOT_INIT = 6, DOM_PILOT = 7, DOM_PROD_INIT = 8, DOM_PROD = 9, DOM_CSPIN = 10, DOM_CBOND = 11,
    DOM_OPTCAL = 12, DOM_PERM = 13
};

static inline uint32_t spin_slot(int i) { return (uint32_t)(((i >> 7) << 5) | (i & 31)); }
static inline int spin_word(int i) { return (i >> 5) & 3; }

static uint32_t draw(uint64_t key64, uint32_t c0, uint32_t c1, uint32_t c2, uint32_t c3, int w) {
    uint32_t ctr[4] = {c0, c1, c2, c3};
    uint32_t key[2] = {(uint32_t)key64, (uint32_t)(key64 >> 32)};
    uint32_t out[4];
    or_philox(ctr, key, out);
    return out[w];
}

static inline float u01(uint32_t x) { return (float)(x >> 8) * (1.0f / 16777216.0f); }

/* Deterministic float32 e^y for y in (-17, 0]: y*log2(e) split into a nearest
 * integer k and a remainder f in [-1/2, 1/2], 2^f by its Taylor series
 * (coefficients ln2^n/n!, n <= 6, Horner with fmaf), 2^k applied to the
 * exponent field.  Single IEEE-rounded operations throughout. */
OR_EXPORT float or_expf(float y) {
    float t = y * 1.44269504f;
    float kf = rintf(t);
    int k = (int)kf;
    float f = t - kf;
    float p = fmaf(1.5403530e-4f, f, 1.3333558e-3f);
    p = fmaf(p, f, 9.6181291e-3f);
    p = fmaf(p, f, 5.5504109e-2f);
    p = fmaf(p, f, 2.4022651e-1f);
    p = fmaf(p, f, 6.9314718e-1f);
    p = fmaf(p, f, 1.0f);
    uint32_t b;
    memcpy(&b, &p, 4);
    b += (uint32_t)k << 23;
    memcpy(&p, &b, 4);
    return p;
}

/* The Metropolis decision of the replay model.  y = -dE (float32), u uniform:
 * qanneal accepts iff dE <= 0 || u < exp(-dE) (annealer.cpp:55,
 * sqa_annealer.cpp:198).  Moves with y <= -17 are rejected outright:
 * exp(-17) = 4.1e-8 is already below the finest step of u (2^-24 = 6.0e-8). */
static inline int metropolis(float y, float u) { return y >= 0.0f || (y > -17.0f && u < or_expf(y)); }

/* ------------------------------------------------------------------ */
/* Models                                                               */
/* ------------------------------------------------------------------ */
enum { M_DENSE = 0, M_SPARSE = 1, M_HUBO = 2 };

typedef struct {
    int kind, n;
    double c;
    double *h64;
    float *h32;
    /* dense: coupling of (i,j) is J[min][max] (the upper triangle, as the
       energy of dense_ising.cpp:29-44 reads it), float32, zero diagonal */
    double *J64;
    float *J32;
    /* sparse: merged adjacency CSR (both directions) + the original edge list */
    int *rowptr, *col;
    float *val32;
    int m;
    int64_t *ei, *ej;
    double *ew;
    /* hubo: consolidated terms (degree >= 2) + incidence lists */
    int T;
    int *tptr, *tvars;
    double *tcoef64;
    float *tcoef32;
    int *incptr, *incterm;
} or_model;

OR_EXPORT void or_model_free(or_model *M) {
    if (!M) return;
    free(M->h64); free(M->h32); free(M->J64); free(M->J32);
    free(M->rowptr); free(M->col); free(M->val32); free(M->ei); free(M->ej); free(M->ew);
    free(M->tptr); free(M->tvars); free(M->tcoef64); free(M->tcoef32);
    free(M->incptr); free(M->incterm);
    free(M);
}

static or_model *model_alloc(int kind, int n, double c) {
    or_model *M = (or_model *)calloc(1, sizeof(or_model));
    M->kind = kind; M->n = n; M->c = c;
    M->h64 = (double *)calloc((size_t)n, sizeof(double));
    M->h32 = (float *)calloc((size_t)n, sizeof(float));
    return M;
}

OR_EXPORT or_model *or_model_dense(int n, const double *h, const double *J, double c) {
    if (n <= 0) return NULL;
    or_model *M = model_alloc(M_DENSE, n, c);
    M->J64 = (double *)malloc((size_t)n * n * sizeof(double));
    M->J32 = (float *)calloc((size_t)n * n, sizeof(float));
    memcpy(M->J64, J, (size_t)n * n * sizeof(double));
    for (int i = 0; i < n; ++i) { M->h64[i] = h[i]; M->h32[i] = (float)h[i]; }
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) {
            if (i == j) continue;
            int a = i < j ? i : j, b = i < j ? j : i;
            M->J32[(size_t)i * n + j] = (float)J[(size_t)a * n + b];
        }
    return M;
}

typedef struct { int nb; double w; int order; } nbr_t;
static int nbr_cmp(const void *a, const void *b) {
    const nbr_t *x = (const nbr_t *)a, *y = (const nbr_t *)b;
    if (x->nb != y->nb) return x->nb < y->nb ? -1 : 1;
    return x->order < y->order ? -1 : (x->order > y->order);
}

OR_EXPORT or_model *or_model_sparse(int n, const double *h, int m, const int64_t *ei, const int64_t *ej,
                                    const double *w, double c) {
    if (n <= 0) return NULL;
    for (int e = 0; e < m; ++e) {
        if (ei[e] < 0 || ej[e] < 0 || ei[e] >= n || ej[e] >= n || ei[e] == ej[e]) return NULL;
    }
    or_model *M = model_alloc(M_SPARSE, n, c);
    for (int i = 0; i < n; ++i) { M->h64[i] = h[i]; M->h32[i] = (float)h[i]; }
    M->m = m;
    M->ei = (int64_t *)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
    M->ej = (int64_t *)malloc(sizeof(int64_t) * (size_t)(m ? m : 1));
    M->ew = (double *)malloc(sizeof(double) * (size_t)(m ? m : 1));
    if (m) {
        memcpy(M->ei, ei, sizeof(int64_t) * m);
        memcpy(M->ej, ej, sizeof(int64_t) * m);
        memcpy(M->ew, w, sizeof(double) * m);
    }
    /* adjacency entries in insertion order (sparse_ising.cpp:35-41), then
       duplicates of one neighbour merged in float64 in that order */
    int *deg = (int *)calloc((size_t)n + 1, sizeof(int));
    for (int e = 0; e < m; ++e) { deg[ei[e]]++; deg[ej[e]]++; }
    int *start = (int *)calloc((size_t)n + 1, sizeof(int));
    for (int i = 0; i < n; ++i) start[i + 1] = start[i] + deg[i];
    nbr_t *tmp = (nbr_t *)malloc(sizeof(nbr_t) * (size_t)(2 * m + 1));
    int *fill = (int *)calloc((size_t)n, sizeof(int));
    for (int e = 0; e < m; ++e) {
        int a = (int)ei[e], b = (int)ej[e];
        tmp[start[a] + fill[a]] = (nbr_t){b, w[e], fill[a]}; fill[a]++;
        tmp[start[b] + fill[b]] = (nbr_t){a, w[e], fill[b]}; fill[b]++;
    }
    M->rowptr = (int *)calloc((size_t)n + 1, sizeof(int));
    M->col = (int *)malloc(sizeof(int) * (size_t)(2 * m + 1));
    M->val32 = (float *)malloc(sizeof(float) * (size_t)(2 * m + 1));
    int nnz = 0;
    for (int i = 0; i < n; ++i) {
        qsort(tmp + start[i], (size_t)deg[i], sizeof(nbr_t), nbr_cmp);
        M->rowptr[i] = nnz;
        int k = start[i];
        while (k < start[i] + deg[i]) {
            int nb = tmp[k].nb;
            double acc = 0.0;
            /* float64 sum in insertion order */
            int kk = k;
            while (kk < start[i] + deg[i] && tmp[kk].nb == nb) { acc += tmp[kk].w; ++kk; }
            M->col[nnz] = nb;
            M->val32[nnz] = (float)acc;
            ++nnz;
            k = kk;
        }
    }
    M->rowptr[n] = nnz;
    free(deg); free(start); free(tmp); free(fill);
    return M;
}

/* HUBO consolidation, restating higher_order_ising.cpp:10-90: parity reduction
   of repeated indices, degree 0 -> c, degree 1 -> h, identical supports merged
   (float64 sums in input order), zero coefficients dropped, terms ordered by
   their sorted support (std::map order). */
typedef struct { int deg; int vars_off; double coef; int order; } rawterm_t;
static int *g_sortvars;
static int rawterm_cmp(const void *a, const void *b) {
    const rawterm_t *x = (const rawterm_t *)a, *y = (const rawterm_t *)b;
    int d = x->deg < y->deg ? x->deg : y->deg;
    for (int k = 0; k < d; ++k) {
        int va = g_sortvars[x->vars_off + k], vb = g_sortvars[y->vars_off + k];
        if (va != vb) return va < vb ? -1 : 1;
    }
    if (x->deg != y->deg) return x->deg < y->deg ? -1 : 1;
    return x->order < y->order ? -1 : (x->order > y->order);
}
static int int_cmp(const void *a, const void *b) {
    int x = *(const int *)a, y = *(const int *)b;
    return x < y ? -1 : (x > y);
}

OR_EXPORT or_model *or_model_hubo(int n, int nraw, const int64_t *rptr, const int64_t *rvars,
                                  const double *rcoef, double c) {
    if (n <= 0) return NULL;
    for (int t = 0; t < nraw; ++t)
        for (int64_t k = rptr[t]; k < rptr[t + 1]; ++k)
            if (rvars[k] < 0 || rvars[k] >= n) return NULL;
    or_model *M = model_alloc(M_HUBO, n, c);
    int64_t totv = nraw ? rptr[nraw] : 0;
    int *sv = (int *)malloc(sizeof(int) * (size_t)(totv + 1));
    rawterm_t *rt = (rawterm_t *)malloc(sizeof(rawterm_t) * (size_t)(nraw + 1));
    int nrt = 0, voff = 0;
    int *buf = (int *)malloc(sizeof(int) * (size_t)(totv + 1));
    for (int t = 0; t < nraw; ++t) {
        if (rcoef[t] == 0.0) continue;
        int len = (int)(rptr[t + 1] - rptr[t]);
        for (int k = 0; k < len; ++k) buf[k] = (int)rvars[rptr[t] + k];
        qsort(buf, (size_t)len, sizeof(int), int_cmp);
        int deg = 0, i = 0;
        while (i < len) {
            int j = i;
            while (j < len && buf[j] == buf[i]) ++j;
            if ((j - i) & 1) sv[voff + deg++] = buf[i];
            i = j;
        }
        if (deg == 0) { M->c += rcoef[t]; continue; }
        if (deg == 1) { M->h64[sv[voff]] += rcoef[t]; continue; }
        rt[nrt] = (rawterm_t){deg, voff, rcoef[t], nrt};
        ++nrt;
        voff += deg;
    }
    free(buf);
    for (int i = 0; i < n; ++i) M->h32[i] = (float)M->h64[i];
    g_sortvars = sv;
    qsort(rt, (size_t)nrt, sizeof(rawterm_t), rawterm_cmp);
    M->tptr = (int *)calloc((size_t)nrt + 1, sizeof(int));
    M->tvars = (int *)malloc(sizeof(int) * (size_t)(voff + 1));
    M->tcoef64 = (double *)malloc(sizeof(double) * (size_t)(nrt + 1));
    M->tcoef32 = (float *)malloc(sizeof(float) * (size_t)(nrt + 1));
    int T = 0, tv = 0, k = 0;
    while (k < nrt) {
        int kk = k;
        double acc = 0.0;
        while (kk < nrt && rawterm_cmp(&(rawterm_t){rt[k].deg, rt[k].vars_off, 0, -1},
                                       &(rawterm_t){rt[kk].deg, rt[kk].vars_off, 0, -1}) == 0) {
            acc += rt[kk].coef;
            ++kk;
        }
        if (acc != 0.0) {
            M->tptr[T] = tv;
            for (int v = 0; v < rt[k].deg; ++v) M->tvars[tv++] = sv[rt[k].vars_off + v];
            M->tcoef64[T] = acc;
            M->tcoef32[T] = (float)acc;
            ++T;
        }
        k = kk;
    }
    M->tptr[T] = tv;
    M->T = T;
    free(rt); free(sv);
    /* incidence lists in term order */
    M->incptr = (int *)calloc((size_t)n + 1, sizeof(int));
    for (int t = 0; t < T; ++t)
        for (int q = M->tptr[t]; q < M->tptr[t + 1]; ++q) M->incptr[M->tvars[q] + 1]++;
    for (int i = 0; i < n; ++i) M->incptr[i + 1] += M->incptr[i];
    M->incterm = (int *)malloc(sizeof(int) * (size_t)(M->incptr[n] + 1));
    int *fill = (int *)calloc((size_t)n, sizeof(int));
    for (int t = 0; t < T; ++t)
        for (int q = M->tptr[t]; q < M->tptr[t + 1]; ++q) {
            int v = M->tvars[q];
            M->incterm[M->incptr[v] + fill[v]++] = t;
        }
    free(fill);
    return M;
}

/* Introspection of the consolidated HUBO (for tests). */
OR_EXPORT int or_model_info(const or_model *M, int *n, int *kind, int *T, double *c) {
    *n = M->n; *kind = M->kind; *T = M->T; *c = M->c;
    return 0;
}
OR_EXPORT void or_model_hubo_terms(const or_model *M, int *tptr, int *tvars, double *coef, double *h) {
    memcpy(tptr, M->tptr, sizeof(int) * (size_t)(M->T + 1));
    memcpy(tvars, M->tvars, sizeof(int) * (size_t)M->tptr[M->T]);
    memcpy(coef, M->tcoef64, sizeof(double) * (size_t)M->T);
    memcpy(h, M->h64, sizeof(double) * (size_t)M->n);
}

/* ---- float64 restatements of the reference's own model functions ---- */

/* energy() in the reference's summation order (dense_ising.cpp:29-44,
   sparse_ising.cpp:43-56, higher_order_ising.cpp:92-111) */
OR_EXPORT double or_energy64(const or_model *M, const int8_t *s) {
    const int n = M->n;
    double E = M->c;
    for (int i = 0; i < n; ++i) E += M->h64[i] * (double)s[i];
    if (M->kind == M_DENSE) {
        for (int i = 0; i < n; ++i)
            for (int j = i + 1; j < n; ++j)
                E += M->J64[(size_t)i * n + j] * (double)s[i] * (double)s[j];
    } else if (M->kind == M_SPARSE) {
        for (int e = 0; e < M->m; ++e) E += M->ew[e] * (double)s[M->ei[e]] * (double)s[M->ej[e]];
    } else {
        for (int t = 0; t < M->T; ++t) {
            double p = M->tcoef64[t];
            for (int q = M->tptr[t]; q < M->tptr[t + 1]; ++q) p *= (double)s[M->tvars[q]];
            E += p;
        }
    }
    return E;
}

/* delta_energy() (dense_ising.cpp:46-62, sparse_ising.cpp:58-71,
   higher_order_ising.cpp:113-136), float64, original coefficients */
OR_EXPORT double or_delta_energy64(const or_model *M, const int8_t *s, int flip) {
    const int n = M->n;
    double local = M->h64[flip];
    if (M->kind == M_DENSE) {
        for (int j = 0; j < n; ++j)
            if (j != flip) local += M->J64[(size_t)flip * n + j] * (double)s[j];
    } else if (M->kind == M_SPARSE) {
        for (int e = 0; e < M->m; ++e) {
            if (M->ei[e] == flip) local += M->ew[e] * (double)s[M->ej[e]];
            else if (M->ej[e] == flip) local += M->ew[e] * (double)s[M->ei[e]];
        }
    } else {
        for (int q = M->incptr[flip]; q < M->incptr[flip + 1]; ++q) {
            int t = M->incterm[q];
            double p = M->tcoef64[t];
            for (int k = M->tptr[t]; k < M->tptr[t + 1]; ++k)
                if (M->tvars[k] != flip) p *= (double)s[M->tvars[k]];
            local += p;
        }
    }
    return -2.0 * (double)s[flip] * local;
}

/* ------------------------------------------------------------------ */
/* Replay-model field cache (float32 g = J.s, h kept apart)            */
/* ------------------------------------------------------------------ */
static void fields_init(const or_model *M, const int8_t *s, float *g) {
    const int n = M->n;
    if (M->kind == M_DENSE) {
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            const float *row = M->J32 + (size_t)i * n;
            for (int j = 0; j < n; ++j) acc += (double)row[j] * (double)s[j];
            g[i] = (float)acc;
        }
    } else if (M->kind == M_SPARSE) {
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int e = M->rowptr[i]; e < M->rowptr[i + 1]; ++e) acc += (double)M->val32[e] * (double)s[M->col[e]];
            g[i] = (float)acc;
        }
    } else {
        for (int i = 0; i < n; ++i) {
            double acc = 0.0;
            for (int q = M->incptr[i]; q < M->incptr[i + 1]; ++q) {
                int t = M->incterm[q];
                int sg = 1;
                for (int k = M->tptr[t]; k < M->tptr[t + 1]; ++k)
                    if (M->tvars[k] != i) sg *= s[M->tvars[k]];
                acc += (double)M->tcoef32[t] * (double)sg;
            }
            g[i] = (float)acc;
        }
    }
}

OR_EXPORT void or_fields_init(const or_model *M, const int8_t *s, float *g) { fields_init(M, s, g); }

/* After flipping spin j whose old value was so (s already holds the new value). */
static void apply_flip(const or_model *M, const int8_t *s, float *g, int j, int so) {
    const int n = M->n;
    const float cf = so > 0 ? -2.0f : 2.0f;
    if (M->kind == M_DENSE) {
        const float *row = M->J32 + (size_t)j * n;
        for (int m = 0; m < n; ++m)
            if (m != j) g[m] = g[m] + cf * row[m];
    } else if (M->kind == M_SPARSE) {
        for (int e = M->rowptr[j]; e < M->rowptr[j + 1]; ++e) {
            int m = M->col[e];
            g[m] = g[m] + cf * M->val32[e];
        }
    } else {
        /* higher_order_ising.cpp:167-189: each other member v of an incident
           term gains 2 * J_t * prod(new spins) * s_v */
        for (int q = M->incptr[j]; q < M->incptr[j + 1]; ++q) {
            int t = M->incterm[q];
            int sg = 1;
            for (int k = M->tptr[t]; k < M->tptr[t + 1]; ++k) sg *= s[M->tvars[k]];
            float two = 2.0f * M->tcoef32[t];
            for (int k = M->tptr[t]; k < M->tptr[t + 1]; ++k) {
                int v = M->tvars[k];
                if (v == j) continue;
                float d = (sg * s[v] > 0) ? two : -two;
                g[v] = g[v] + d;
            }
        }
    }
}

/* Flip spin i of s (in place) and update the float32 field cache g the way
   the sweeps do (for the field-drift restatement of
   test_higher_order_ising.cpp:149-167). */
OR_EXPORT void or_flip_update(const or_model *M, int8_t *s, float *g, int i) {
    const int so = s[i];
    s[i] = (int8_t)-so;
    apply_flip(M, s, g, i, so);
}

/* float64 sum in warp order: 32 lane-strided partials, then xor butterfly */
static double wsum(const double *v, int n) {
    double p[32];
    for (int l = 0; l < 32; ++l) p[l] = 0.0;
    for (int i = 0; i < n; ++i) p[i & 31] += v[i];
    for (int off = 16; off >= 1; off >>= 1) {
        double q[32];
        for (int l = 0; l < 32; ++l) q[l] = p[l] + p[l ^ off];
        memcpy(p, q, sizeof(p));
    }
    return p[0];
}

/* Tracking energy of one slice from its field cache. */
static double energy_track(const or_model *M, const int8_t *s, const float *g, double *scratch) {
    const int n = M->n;
    for (int i = 0; i < n; ++i) scratch[i] = (double)s[i] * (double)M->h32[i];
    double eh = wsum(scratch, n);
    if (M->kind != M_HUBO) {
        for (int i = 0; i < n; ++i) scratch[i] = (double)s[i] * (double)g[i];
        return M->c + (eh + 0.5 * wsum(scratch, n));
    }
    double *st = scratch + n;
    for (int t = 0; t < M->T; ++t) {
        int sg = 1;
        for (int k = M->tptr[t]; k < M->tptr[t + 1]; ++k) sg *= s[M->tvars[k]];
        st[t] = sg > 0 ? (double)M->tcoef32[t] : -(double)M->tcoef32[t];
    }
    double ej = wsum(st, M->T);
    return M->c + (eh + ej);
}

OR_EXPORT double or_energy_track(const or_model *M, const int8_t *s) {
    float *g = (float *)malloc(sizeof(float) * (size_t)M->n);
    double *sc = (double *)malloc(sizeof(double) * (size_t)(M->n + M->T + 1));
    fields_init(M, s, g);
    double E = energy_track(M, s, g, sc);
    free(g); free(sc);
    return E;
}

static void init_spins(int8_t *s, int n, uint64_t key, uint32_t cell, uint32_t tag) {
    const int nw = (n + 31) / 32;
    for (int q = 0; q < nw; ++q) {
        uint32_t w = draw(key, (uint32_t)(q >> 2), cell, 0u, tag, q & 3);
        for (int b = 0; b < 32 && 32 * q + b < n; ++b) s[32 * q + b] = ((w >> b) & 1u) ? 1 : -1;
    }
}

OR_EXPORT void or_init_spins(int8_t *s, int n, uint64_t key, uint32_t cell, uint32_t tag) {
    init_spins(s, n, key, cell, tag);
}

static double trotter_coupling(double beta, double gamma, int P) {
    double x = beta * gamma / (double)P;
    if (x < 1e-12) x = 1e-12;
    return 0.5 * log(1.0 / tanh(x));
}

/* ------------------------------------------------------------------ */
/* SA (annealer.cpp:33-75)                                              */
/* ------------------------------------------------------------------ */
/* mag_trace (nullable): magnetisation after each step (ReplicaAnnealer,
   replica_annealer.cpp:119-131); best_step (nullable): the step whose sweeps
   last lowered the best energy, -1 for the starting state. */
/* Sweep traces for the observer tests (annealer.cpp:48-71,
   sqa_annealer.cpp:318-473): set before one run, cleared with stride 0.
   SA: the state and running energy after every recorded sweep
   ([steps][rps][n], [steps][rps]), the state at each step end (end_states,
   [steps][n]) and the magnetisation per step.  SQA: per
   ring the bits and slice energies after every recorded sweep
   ([K][steps][rps][P][n], [K][steps][rps][P]; records of a step: slice,
   cluster, worldline sweeps), at the start and each step end
   ([K][steps+1][P][n], [K][steps+1][P]), and the magnetisation over all rings
   per step.  A sweep is recorded when its index in its phase is a multiple
   of stride. */
static struct {
    int stride;
    int8_t *states, *ring_states, *end_states;
    double *energies, *ring_E, *end_E, *mag;
} g_tr;

OR_EXPORT void or_trace_set(int stride, int8_t *states, double *energies, int8_t *ring_states, double *ring_E,
                            int8_t *end_states, double *end_E, double *mag) {
    g_tr.stride = stride;
    g_tr.states = states; g_tr.energies = energies;
    g_tr.ring_states = ring_states; g_tr.ring_E = ring_E;
    g_tr.end_states = end_states; g_tr.end_E = end_E;
    g_tr.mag = mag;
}

static int tr_count(int sweeps) { return g_tr.stride > 0 ? (sweeps + g_tr.stride - 1) / g_tr.stride : 0; }

OR_EXPORT int or_sa_run(const or_model *M, const double *betas, int steps, int spb, uint64_t seed, int read,
                        int8_t *best_spins, double *best_E, double *trace, int64_t *counters, double *mag_trace,
                        int *best_step) {
    const int n = M->n;
    const uint64_t key = seed + (uint64_t)read;
    int8_t *s = (int8_t *)malloc((size_t)n);
    float *g = (float *)malloc(sizeof(float) * (size_t)n);
    double *sc = (double *)malloc(sizeof(double) * (size_t)(n + M->T + 1));
    init_spins(s, n, key, 0u, DOM_INIT);
    fields_init(M, s, g);
    double E = energy_track(M, s, g, sc);
    double best = E;
    int bstep = -1;
    memcpy(best_spins, s, (size_t)n);
    int64_t att = 0, acc = 0;
    for (int step = 0; step < steps; ++step) {
        const float B = (float)(2.0 * betas[step]);
        for (int sw = 0; sw < spb; ++sw) {
            const uint32_t sigma = (uint32_t)(step * spb + sw);
            for (int i = 0; i < n; ++i) {
                float u = u01(draw(key, spin_slot(i), 0u, sigma, DOM_SA, spin_word(i)));
                float loc = M->h32[i] + g[i];
                float x = s[i] > 0 ? loc : -loc;
                ++att;
                if (metropolis(x * B, u)) {
                    ++acc;
                    int so = s[i];
                    double xd = (double)so * ((double)M->h32[i] + (double)g[i]);
                    s[i] = (int8_t)-so;
                    apply_flip(M, s, g, i, so);
                    E += -2.0 * xd;
                    if (E < best) { best = E; bstep = step; memcpy(best_spins, s, (size_t)n); }
                }
            }
            if (g_tr.stride > 0 && sw % g_tr.stride == 0) {
                const size_t rec = (size_t)step * tr_count(spb) + (size_t)(sw / g_tr.stride);
                if (g_tr.states) memcpy(g_tr.states + rec * n, s, (size_t)n);
                if (g_tr.energies) g_tr.energies[rec] = E;
            }
        }
        trace[step] = E;
        if (g_tr.stride > 0 && g_tr.end_states) memcpy(g_tr.end_states + (size_t)step * n, s, (size_t)n);
        if (mag_trace || (g_tr.stride > 0 && g_tr.mag)) {
            long long m = 0;
            for (int i = 0; i < n; ++i) m += s[i];
            if (mag_trace) mag_trace[step] = (double)m / (double)n;
            if (g_tr.stride > 0 && g_tr.mag) g_tr.mag[step] = (double)m / (double)n;
        }
    }
    *best_E = best;
    if (best_step) *best_step = bstep;
    if (counters) { counters[0] = att; counters[1] = acc; }
    free(s); free(g); free(sc);
    return 0;
}

/* ------------------------------------------------------------------ */
/* Trotter ring sweeps shared by SQA, SQA-PT and SQA-Chi                */
/* ------------------------------------------------------------------ */
typedef struct {
    const or_model *M;
    int n, P, K;
    int8_t *s;   /* [K*P][n] */
    float *g;    /* [K*P][n] */
    double *sc;
    uint64_t key;
    int64_t att_slice, acc_slice, att_world, acc_world;
} ring_t;

static int phase_of(int t, int P) {
    if ((P & 1) && t == P - 1) return 2;
    return t & 1;
}

/* Update order of the SQA and SQA-PT sweeps (the SQA-Chi kernel keeps its own
   parity checkerboard, sqa_chi_annealer.cpp:68-140, in every mode):
   1 (default): qanneal's order in law -- before every slice, cluster and
     worldline sweep a fresh uniformly random spin order (std::shuffle at
     sqa_annealer.cpp:181,216,295,599,631,703 and
     sqa_parallel_tempering.cpp:209,224,281,489), the slices of a ring swept
     one after another, t = 0 .. P-1, each in that order;
   0: parity checkerboard over the slices (even, odd, the last odd one alone),
     spins ascending. */
static int g_order = 1;
OR_EXPORT void or_set_update_order(int order) { g_order = order ? 1 : 0; }
OR_EXPORT int or_get_update_order(void) { return g_order; }

static int u64_cmp(const void *a, const void *b) {
    const uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return x < y ? -1 : (x > y ? 1 : 0);
}

/* The random spin order of one sweep: spins sorted by the 64-bit keys
   K_i = (r_i with its low 20 bits cleared) | i, r_i = (x_a << 32) | x_b from
   philox(i >> 1, ring, sweep, (tag << 8) | DOM_PERM) -- words 0, 1 for even
   i, words 2, 3 for odd i.  44 random bits a key make ties (broken by the
   spin index) negligible, so the order is uniform over all n! orders, as
   std::shuffle's.  order[p] is the spin visited p-th. */
static void sweep_order(uint64_t key, uint32_t ring, uint32_t sigma, uint32_t tag, int n, int *order) {
    uint64_t *K = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)n);
    uint32_t out[4] = {0, 0, 0, 0};
    for (int i = 0; i < n; ++i) {
        if ((i & 1) == 0) {
            uint32_t ctr[4] = {(uint32_t)(i >> 1), ring, sigma, (tag << 8) | DOM_PERM};
            uint32_t kk[2] = {(uint32_t)key, (uint32_t)(key >> 32)};
            or_philox(ctr, kk, out);
        }
        const uint64_t r = ((uint64_t)out[2 * (i & 1)] << 32) | out[2 * (i & 1) + 1];
        K[i] = (r & ~(uint64_t)0xFFFFF) | (uint64_t)i;
    }
    qsort(K, (size_t)n, sizeof(uint64_t), u64_cmp);
    for (int p = 0; p < n; ++p) order[p] = (int)(K[p] & 0xFFFFF);
    free(K);
}

OR_EXPORT void or_sweep_order(uint64_t key, uint32_t ring, uint32_t sigma, uint32_t tag, int n, int *order) {
    sweep_order(key, ring, sigma, tag, n, order);
}

static void ring_alloc(ring_t *R, const or_model *M, int P, int K, uint64_t key) {
    memset(R, 0, sizeof(*R));
    R->M = M; R->n = M->n; R->P = P; R->K = K; R->key = key;
    R->s = (int8_t *)malloc((size_t)K * P * M->n);
    R->g = (float *)malloc(sizeof(float) * (size_t)K * P * M->n);
    R->sc = (double *)malloc(sizeof(double) * (size_t)(M->n + M->T + 1));
}
static void ring_free(ring_t *R) { free(R->s); free(R->g); free(R->sc); }

static void ring_init(ring_t *R, uint32_t tag) {
    for (int c = 0; c < R->K * R->P; ++c) {
        init_spins(R->s + (size_t)c * R->n, R->n, R->key, (uint32_t)c, tag);
        fields_init(R->M, R->s + (size_t)c * R->n, R->g + (size_t)c * R->n);
    }
}

/* One slice of one ring: sqa_annealer.cpp:180-209 / sqa_chi_annealer.cpp:96-121.
   rng_cell is the cell index used in the counter (ring-relative k*P+t unless
   a slot remap applies). */
static void sweep_cell_ord(ring_t *R, int k, int t, uint32_t rng_cell, uint32_t sigma, uint32_t tag, float B,
                           float T4, const int *order) {
    const or_model *M = R->M;
    const int n = R->n, P = R->P;
    const int prev = t == 0 ? P - 1 : t - 1, next = (t + 1) % P;
    int8_t *s = R->s + ((size_t)k * P + t) * n;
    const int8_t *sp = R->s + ((size_t)k * P + prev) * n;
    const int8_t *sn = R->s + ((size_t)k * P + next) * n;
    float *g = R->g + ((size_t)k * P + t) * n;
    for (int pos = 0; pos < n; ++pos) {
        /* the uniform belongs to the visiting position, the spin to the order */
        const int i = order ? order[pos] : pos;
        const int si = s[i];
        const int q = si * (sp[i] + sn[i]) / 2;
        const float tro = q == 0 ? 0.0f : (q > 0 ? T4 : -T4);
        float u = u01(draw(R->key, spin_slot(pos), rng_cell, sigma, tag, spin_word(pos)));
        float loc = M->h32[i] + g[i];
        float x = si > 0 ? loc : -loc;
        R->att_slice++;
        if (metropolis(x * B - tro, u)) {
            R->acc_slice++;
            s[i] = (int8_t)-si;
            apply_flip(M, s, g, i, si);
        }
    }
}

static void sweep_cell(ring_t *R, int k, int t, uint32_t rng_cell, uint32_t sigma, uint32_t tag, float B, float T4) {
    sweep_cell_ord(R, k, t, rng_cell, sigma, tag, B, T4, NULL);
}

/* One slice sweep of ring k in qanneal's order: one random spin order for the
   sweep, slices t = 0 .. P-1 in turn (sqa_annealer.cpp:180-209,
   sqa_parallel_tempering.cpp:208-221).  B and T4 may differ per ring (PT). */
static void ring_slice_sweep_ref(ring_t *R, int k, uint32_t slot, uint32_t sigma, uint32_t tag, float B, float T4) {
    int *order = (int *)malloc(sizeof(int) * (size_t)R->n);
    sweep_order(R->key, slot, sigma, tag, R->n, order);
    for (int t = 0; t < R->P; ++t) sweep_cell_ord(R, k, t, slot * (uint32_t)R->P + (uint32_t)t, sigma, tag, B, T4, order);
    free(order);
}

/* The parity checkerboard (SQA-Chi's order, and the opt-in order of SQA / SQA-PT). */
static void slice_sweep_cb(ring_t *R, uint32_t sigma, uint32_t tag, float B, float T4, const int *slot_of_ring) {
    for (int ph = 0; ph < 3; ++ph)
        for (int k = 0; k < R->K; ++k)
            for (int t = 0; t < R->P; ++t) {
                if (phase_of(t, R->P) != ph) continue;
                int slot = slot_of_ring ? slot_of_ring[k] : k;
                sweep_cell(R, k, t, (uint32_t)(slot * R->P + t), sigma, tag, B, T4);
            }
}

static void slice_sweep(ring_t *R, uint32_t sigma, uint32_t tag, float B, float T4, const int *slot_of_ring) {
    if (!g_order) {
        slice_sweep_cb(R, sigma, tag, B, T4, slot_of_ring);
        return;
    }
    for (int k = 0; k < R->K; ++k)
        ring_slice_sweep_ref(R, k, (uint32_t)(slot_of_ring ? slot_of_ring[k] : k), sigma, tag, B, T4);
}

/* sqa_annealer.cpp:294-315 */
static void worldline_sweep(ring_t *R, int k, uint32_t rng_ring, uint32_t sigma, float B) {
    const or_model *M = R->M;
    const int n = R->n, P = R->P;
    int *order = NULL;
    if (g_order) {
        order = (int *)malloc(sizeof(int) * (size_t)n);
        sweep_order(R->key, rng_ring, sigma, DOM_WORLD, n, order);
    }
    for (int pos = 0; pos < n; ++pos) {
        const int i = order ? order[pos] : pos;
        int sh = 0;
        double G = 0.0;
        for (int t = 0; t < P; ++t) {
            int st = R->s[((size_t)k * P + t) * n + i];
            sh += st;
            G += (double)st * (double)R->g[((size_t)k * P + t) * n + i];
        }
        float x = (float)((double)M->h32[i] * (double)sh + G);
        float u = u01(draw(R->key, spin_slot(pos), rng_ring, sigma, DOM_WORLD, spin_word(pos)));
        R->att_world++;
        if (metropolis(x * B, u)) {
            R->acc_world++;
            for (int t = 0; t < P; ++t) {
                int8_t *s = R->s + ((size_t)k * P + t) * n;
                int so = s[i];
                s[i] = (int8_t)-so;
                apply_flip(M, s, R->g + ((size_t)k * P + t) * n, i, so);
            }
        }
    }
    free(order);
}

/* Cluster move of spin i of replica k along imaginary time, the
   Swendsen-Wang step of sqa_annealer.cpp:215-288 (and
   sqa_parallel_tempering.cpp:224-278) in the replay form:
   - seed slice t0 = floor(u * P) from word 0 of philox(0, ring, sweep,
     CSPIN | i << 8); the acceptance uniform is word 1 of the same call;
   - bond b joins slices b and b+1 (mod P) when both carry the seed's spin and
     its uniform (word b & 3 of philox(b >> 2, ring, sweep, CBOND | i << 8))
     is below JP = 1 - exp(-2 J_perp); the cluster is the run of joined bonds
     through t0, grown right then left (every slice when the run closes the
     ring, as the reference's growth does with P - 1 joined bonds);
   - y = x B - k T4 / 2 with x = h s0 |C| + sum_{t in C} s0 g_t (the sum in
     warp order over t) and k = s0 (s_left + s_right) over the two slices
     just outside the cluster (none when it is the whole ring). */
static int cluster_move(ring_t *R, int k, int i, uint32_t rng_ring, uint32_t sigma, float B, float T4, float JP) {
    const or_model *M = R->M;
    const int n = R->n, P = R->P;
    int8_t *s = R->s + (size_t)k * P * n;
    float *g = R->g + (size_t)k * P * n;
    const uint32_t c3s = DOM_CSPIN | ((uint32_t)i << 8), c3b = DOM_CBOND | ((uint32_t)i << 8);
    const int t0 = (int)(((uint64_t)(draw(R->key, 0u, rng_ring, sigma, c3s, 0) >> 8) * (uint64_t)P) >> 24);
    const float u = u01(draw(R->key, 0u, rng_ring, sigma, c3s, 1));
    const int s0 = s[(size_t)t0 * n + i];
    int act[64];
    int all = 1;
    for (int b = 0; b < P; ++b) {
        const int b1 = b + 1 == P ? 0 : b + 1;
        act[b] = s[(size_t)b * n + i] == s0 && s[(size_t)b1 * n + i] == s0 &&
                 u01(draw(R->key, (uint32_t)(b >> 2), rng_ring, sigma, c3b, b & 3)) < JP;
        all &= act[b];
    }
    int inC[64] = {0};
    int kb = 0, r = 0, l = 0;
    if (!all) {
        while (act[(t0 + r) % P]) ++r;
        while (act[((t0 - 1 - l) % P + P) % P]) ++l;
        all = l + r + 1 >= P;  /* the arc closes on itself: every slice, no boundary */
    }
    if (all) {
        for (int t = 0; t < P; ++t) inC[t] = 1;
    } else {
        for (int d = -l; d <= r; ++d) inC[((t0 + d) % P + P) % P] = 1;
        const int tl = ((t0 - l - 1) % P + P) % P, tr = (t0 + r + 1) % P;
        kb = s0 * s[(size_t)tl * n + i] + s0 * s[(size_t)tr * n + i];
    }
    double c[64];
    int size = 0;
    for (int t = 0; t < P; ++t) {
        c[t] = inC[t] ? (double)s0 * (double)g[(size_t)t * n + i] : 0.0;
        size += inC[t];
    }
    const double G = wsum(c, P);
    const float x = (float)((double)M->h32[i] * (double)(s0 * size) + G);
    const float y = (x * B) - ((float)kb * (0.5f * T4));
    if (!metropolis(y, u)) return 0;
    for (int t = 0; t < P; ++t)
        if (inC[t]) {
            int8_t *st = s + (size_t)t * n;
            st[i] = (int8_t)-s0;
            apply_flip(M, st, g + (size_t)t * n, i, s0);
        }
    return 1;
}

static void cluster_sweep(ring_t *R, int k, uint32_t rng_ring, uint32_t sigma, float B, float T4, float JP) {
    if (!g_order) {
        for (int i = 0; i < R->n; ++i) cluster_move(R, k, i, rng_ring, sigma, B, T4, JP);
        return;
    }
    int *order = (int *)malloc(sizeof(int) * (size_t)R->n);
    sweep_order(R->key, rng_ring, sigma, DOM_CSPIN, R->n, order);
    for (int p = 0; p < R->n; ++p) cluster_move(R, k, order[p], rng_ring, sigma, B, T4, JP);
    free(order);
}

static float join_prob(double beta, double gamma, int P) {
    return (float)(1.0 - exp(-2.0 * trotter_coupling(beta, gamma, P)));
}

static double cell_energy(ring_t *R, int c) {
    return energy_track(R->M, R->s + (size_t)c * R->n, R->g + (size_t)c * R->n, R->sc);
}

/* Per-step constants: beta_scale = beta/P, B = 2 beta_scale, T4 = 4 J_perp. */
static void step_consts(double beta, double gamma, int P, float *B, float *T4) {
    const double bs = beta / (double)P;
    *B = (float)(2.0 * bs);
    *T4 = (float)(4.0 * trotter_coupling(beta, gamma, P));
}

/* ------------------------------------------------------------------ */
/* SQA run (sqa_annealer.cpp:87-477), one read                          */
/* ------------------------------------------------------------------ */
OR_EXPORT int or_sqa_run(const or_model *M, const double *betas, const double *gammas, int steps, int P, int K,
                         int spb, int wls, uint64_t seed, int read, int8_t *best_spins, double *best_E,
                         double *trace, int64_t *counters, int cls) {
    const int n = M->n;
    ring_t R;
    ring_alloc(&R, M, P, K, seed + (uint64_t)read);
    ring_init(&R, DOM_INIT);
    double *rbest = (double *)malloc(sizeof(double) * (size_t)K);
    int *rstep = (int *)malloc(sizeof(int) * (size_t)K);
    int8_t *rstate = (int8_t *)malloc((size_t)K * n);
    double *rsum = (double *)malloc(sizeof(double) * (size_t)K);
    for (int k = 0; k < K; ++k) { rbest[k] = INFINITY; rstep[k] = -1; }
    const int tr_s = tr_count(spb), tr_c = tr_count(cls), rps = tr_s + tr_c + tr_count(wls);
    /* ring k's bits and slice energies into trace record rec (of records of P*n and P) */
    #define TR_RING(STATES, ENERGIES, K_, REC)                                                       \
        do {                                                                                         \
            const size_t rec_ = (REC);                                                               \
            if (STATES) memcpy((STATES) + rec_ * P * n, R.s + (size_t)(K_) * P * n, (size_t)P * n);  \
            if (ENERGIES)                                                                            \
                for (int t_ = 0; t_ < P; ++t_) (ENERGIES)[rec_ * P + t_] = cell_energy(&R, (K_) * P + t_); \
        } while (0)
    if (g_tr.stride > 0)
        for (int k = 0; k < K; ++k) TR_RING(g_tr.end_states, g_tr.end_E, k, (size_t)k * (steps + 1));
    for (int step = 0; step < steps; ++step) {
        float B, T4;
        step_consts(betas[step], gammas[step], P, &B, &T4);
        for (int sw = 0; sw < spb; ++sw) {
            slice_sweep(&R, (uint32_t)(step * spb + sw), DOM_SLICE, B, T4, NULL);
            if (g_tr.stride > 0 && sw % g_tr.stride == 0)
                for (int k = 0; k < K; ++k)
                    TR_RING(g_tr.ring_states, g_tr.ring_E, k,
                            ((size_t)k * steps + step) * rps + (size_t)(sw / g_tr.stride));
        }
        if (cls > 0) {
            const float JP = join_prob(betas[step], gammas[step], P);
            for (int sw = 0; sw < cls; ++sw)
                for (int k = 0; k < K; ++k) {
                    cluster_sweep(&R, k, (uint32_t)k, (uint32_t)(step * cls + sw), B, T4, JP);
                    if (g_tr.stride > 0 && sw % g_tr.stride == 0)
                        TR_RING(g_tr.ring_states, g_tr.ring_E, k,
                                ((size_t)k * steps + step) * rps + (size_t)(tr_s + sw / g_tr.stride));
                }
        }
        for (int sw = 0; sw < wls; ++sw)
            for (int k = 0; k < K; ++k) {
                worldline_sweep(&R, k, (uint32_t)k, (uint32_t)(step * wls + sw), B);
                if (g_tr.stride > 0 && sw % g_tr.stride == 0)
                    TR_RING(g_tr.ring_states, g_tr.ring_E, k,
                            ((size_t)k * steps + step) * rps + (size_t)(tr_s + tr_c + sw / g_tr.stride));
            }
        if (g_tr.stride > 0) {
            long long m = 0;
            for (size_t c = 0; c < (size_t)K * P * n; ++c) m += R.s[c];
            if (g_tr.mag) g_tr.mag[step] = (double)m / (double)((size_t)K * P * n);
            for (int k = 0; k < K; ++k)
                TR_RING(g_tr.end_states, g_tr.end_E, k, (size_t)k * (steps + 1) + step + 1);
        }
        for (int k = 0; k < K; ++k) {
            double sum = 0.0, emin = INFINITY;
            int tmin = 0;
            for (int t = 0; t < P; ++t) {
                double E = cell_energy(&R, k * P + t);
                sum += E;
                if (E < emin) { emin = E; tmin = t; }
            }
            rsum[k] = sum;
            if (emin < rbest[k]) {
                rbest[k] = emin; rstep[k] = step;
                memcpy(rstate + (size_t)k * n, R.s + ((size_t)k * P + tmin) * n, (size_t)n);
            }
        }
        double tot = 0.0;
        for (int k = 0; k < K; ++k) tot += rsum[k];
        trace[step] = tot / (double)(K * P);
    }
    int kb = 0;
    for (int k = 1; k < K; ++k)
        if (rbest[k] < rbest[kb] || (rbest[k] == rbest[kb] && rstep[k] < rstep[kb])) kb = k;
    *best_E = rbest[kb];
    memcpy(best_spins, rstate + (size_t)kb * n, (size_t)n);
    if (counters) {
        counters[0] = R.att_slice; counters[1] = R.acc_slice;
        counters[2] = R.att_world; counters[3] = R.acc_world;
    }
    free(rbest); free(rstep); free(rstate); free(rsum);
    ring_free(&R);
    return 0;
}

#undef TR_RING

/* Step-end scan of one ring: sum and minimum of the slice energies, the
   slice of the minimum, and the imaginary-time bond sum
   B = sum_t sum_i s_t,i s_t+1,i (sqa_parallel_tempering.cpp:128-170). */
static void ring_scan(ring_t *R, int k, double *sum, double *emin, int *tmin, long long *bond) {
    const int n = R->n, P = R->P;
    double s = 0.0, em = INFINITY;
    int tm = 0;
    for (int t = 0; t < P; ++t) {
        double E = cell_energy(R, k * P + t);
        s += E;
        if (E < em) { em = E; tm = t; }
    }
    long long b = 0;
    for (int t = 0; t < P; ++t) {
        const int8_t *a = R->s + ((size_t)k * P + t) * n;
        const int8_t *c = R->s + ((size_t)k * P + (t + 1) % P) * n;
        for (int i = 0; i < n; ++i) b += a[i] * c[i];
    }
    *sum = s; *emin = em; *tmin = tm; *bond = b;
}

/* ------------------------------------------------------------------ */
/* SQA parallel tempering (sqa_parallel_tempering.cpp:81-346), one read  */
/* Rung r ("slot") keeps its (beta_r, Gamma_r) and its random streams;   */
/* swaps exchange which ring sits in which slot, pairs r = 0..R-2 in     */
/* order (cascading), every swap_interval steps.                         */
/* ------------------------------------------------------------------ */
static int sqapt_core(const or_model *M, const double *betas, const double *gammas, int Rn, int P, int spb, int wls,
                      int steps, int swap_interval, uint64_t seed, int read, int8_t *best_spins, double *best_E,
                      double *final_E, int8_t *final_spins, double *avg_trace, double *swap_trace,
                      int64_t *counters, int cls, int classical);

OR_EXPORT int or_sqapt_run(const or_model *M, const double *betas, const double *gammas, int Rn, int P, int spb,
                           int wls, int steps, int swap_interval, uint64_t seed, int read, int8_t *best_spins,
                           double *best_E, double *final_E, int8_t *final_spins, double *avg_trace,
                           double *swap_trace, int64_t *counters, int cls) {
    return sqapt_core(M, betas, gammas, Rn, P, spb, wls, steps, swap_interval, seed, read, best_spins, best_E,
                      final_E, final_spins, avg_trace, swap_trace, counters, cls, 0);
}

/* Classical parallel tempering (parallel_tempering.cpp:36-122): the SQA-PT
   core with one slice per rung and no transverse field -- B = 2 beta, no
   Trotter term, the swap action beta E, so a swap of rungs i, i+1 is
   accepted on -(beta_i - beta_{i+1}) (E_{i+1} - E_i) -- and no worldline or
   cluster moves. */
OR_EXPORT int or_pt_run(const or_model *M, const double *betas, int Rn, int spb, int steps, int swap_interval,
                        uint64_t seed, int read, int8_t *best_spins, double *best_E, double *final_E,
                        int8_t *final_spins, double *avg_trace, double *swap_trace, int64_t *counters) {
    return sqapt_core(M, betas, betas, Rn, 1, spb, 0, steps, swap_interval, seed, read, best_spins, best_E, final_E,
                      final_spins, avg_trace, swap_trace, counters, 0, 1);
}

static int sqapt_core(const or_model *M, const double *betas, const double *gammas, int Rn, int P, int spb, int wls,
                      int steps, int swap_interval, uint64_t seed, int read, int8_t *best_spins, double *best_E,
                      double *final_E, int8_t *final_spins, double *avg_trace, double *swap_trace,
                      int64_t *counters, int cls, int classical) {
    const int n = M->n;
    ring_t R;
    ring_alloc(&R, M, P, Rn, seed + (uint64_t)read);
    ring_init(&R, DOM_INIT);
    int *slot_of = (int *)malloc(sizeof(int) * (size_t)Rn), *ring_in = (int *)malloc(sizeof(int) * (size_t)Rn);
    float *B = (float *)malloc(sizeof(float) * (size_t)Rn), *T4 = (float *)malloc(sizeof(float) * (size_t)Rn);
    double *bp = (double *)malloc(sizeof(double) * (size_t)Rn), *jp = (double *)malloc(sizeof(double) * (size_t)Rn);
    double *Esum = (double *)malloc(sizeof(double) * (size_t)Rn), *Emin = (double *)malloc(sizeof(double) * (size_t)Rn);
    int *tmin = (int *)malloc(sizeof(int) * (size_t)Rn);
    long long *bond = (long long *)malloc(sizeof(long long) * (size_t)Rn);
    for (int k = 0; k < Rn; ++k) {
        slot_of[k] = ring_in[k] = k;
        step_consts(betas[k], gammas[k], P, &B[k], &T4[k]);
        bp[k] = betas[k] / (double)P;
        jp[k] = trotter_coupling(betas[k], gammas[k], P);
        if (classical) { T4[k] = 0.0f; jp[k] = 0.0; }
    }
    double best = INFINITY;
    for (int k = 0; k < Rn; ++k) ring_scan(&R, k, &Esum[k], &Emin[k], &tmin[k], &bond[k]);
    for (int r = 0; r < Rn; ++r) {
        const int k = ring_in[r];
        if (Emin[k] < best) {
            best = Emin[k];
            memcpy(best_spins, R.s + ((size_t)k * P + tmin[k]) * n, (size_t)n);
        }
    }
    for (int step = 0; step < steps; ++step) {
        for (int sw = 0; sw < spb; ++sw) {
            const uint32_t sigma = (uint32_t)(step * spb + sw);
            if (g_order && !classical)  /* classical PT: ascending (parallel_tempering.cpp:36-122) */
                for (int k = 0; k < Rn; ++k)
                    ring_slice_sweep_ref(&R, k, (uint32_t)slot_of[k], sigma, DOM_SLICE, B[slot_of[k]], T4[slot_of[k]]);
            else
                for (int ph = 0; ph < 3; ++ph)
                    for (int k = 0; k < Rn; ++k)
                        for (int t = 0; t < P; ++t) {
                            if (phase_of(t, P) != ph) continue;
                            const int sl = slot_of[k];
                            sweep_cell(&R, k, t, (uint32_t)(sl * P + t), sigma, DOM_SLICE, B[sl], T4[sl]);
                        }
        }
        for (int sw = 0; sw < cls; ++sw)
            for (int k = 0; k < Rn; ++k) {
                const int sl = slot_of[k];
                cluster_sweep(&R, k, (uint32_t)sl, (uint32_t)(step * cls + sw), B[sl], T4[sl],
                              join_prob(betas[sl], gammas[sl], P));
            }
        for (int sw = 0; sw < wls; ++sw)
            for (int k = 0; k < Rn; ++k)
                worldline_sweep(&R, k, (uint32_t)slot_of[k], (uint32_t)(step * wls + sw), B[slot_of[k]]);
        for (int k = 0; k < Rn; ++k) ring_scan(&R, k, &Esum[k], &Emin[k], &tmin[k], &bond[k]);
        for (int r = 0; r < Rn; ++r) {
            const int k = ring_in[r];
            if (Emin[k] < best) {
                best = Emin[k];
                memcpy(best_spins, R.s + ((size_t)k * P + tmin[k]) * n, (size_t)n);
            }
        }
        double acc = 0.0, att = 0.0;
        if ((step + 1) % swap_interval == 0) {
            const uint32_t w = (uint32_t)((step + 1) / swap_interval - 1);
            for (int r = 0; r + 1 < Rn; ++r) {
                const int a = ring_in[r], b = ring_in[r + 1];
                const double e_aa = bp[r] * Esum[a] - jp[r] * (double)bond[a];
                const double e_bb = bp[r + 1] * Esum[b] - jp[r + 1] * (double)bond[b];
                const double e_ab = bp[r] * Esum[b] - jp[r] * (double)bond[b];
                const double e_ba = bp[r + 1] * Esum[a] - jp[r + 1] * (double)bond[a];
                const double delta = (e_ab + e_ba) - (e_aa + e_bb);
                att += 1.0;
                const float u = u01(draw(R.key, (uint32_t)r, 0u, w, DOM_SWAP, 0));
                if (metropolis((float)(-delta), u)) {
                    ring_in[r] = b;
                    ring_in[r + 1] = a;
                    slot_of[b] = r;
                    slot_of[a] = r + 1;
                    acc += 1.0;
                }
            }
        }
        double avg = 0.0;
        for (int r = 0; r < Rn; ++r) avg += Emin[ring_in[r]];
        avg_trace[step] = avg / (double)Rn;
        swap_trace[step] = att > 0.0 ? acc / att : 0.0;
    }
    for (int r = 0; r < Rn; ++r) {
        const int k = ring_in[r];
        final_E[r] = Emin[k];
        memcpy(final_spins + (size_t)r * n, R.s + ((size_t)k * P + tmin[k]) * n, (size_t)n);
    }
    *best_E = best;
    if (counters) {
        counters[0] = R.att_slice; counters[1] = R.acc_slice;
        counters[2] = R.att_world; counters[3] = R.acc_world;
    }
    free(slot_of); free(ring_in); free(B); free(T4); free(bp); free(jp); free(Esum); free(Emin); free(tmin); free(bond);
    ring_free(&R);
    return 0;
}

/* ------------------------------------------------------------------ */
/* SQA-Chi (sqa_chi_annealer.cpp:146-438), one read                     */
/* ------------------------------------------------------------------ */
static double chi_s_to_gamma(double A0, double s) {
    s = s < 1e-10 ? 1e-10 : s;
    s = s > 1.0 - 1e-10 ? 1.0 - 1e-10 : s;
    return A0 * (1.0 - s) / s;
}

/* Stage 2 (sqa_chi_annealer.cpp:283-387): the chi_B peak, the floor, the
   4096-point trapezoid CDF of w(s) = max(chi_B(s), floor) and its inverse at
   uniform targets, and the phase-1 beta ramp.  scalars = {s*, Gamma*, J_perp*,
   floor}. */
OR_EXPORT void or_chi_schedule(int Pts, const double *scan_s, const double *scan_gamma, const double *chi,
                               double beta, double gamma_start, double gamma_end, double A0, int slices,
                               int num_steps, double chi_floor_fraction, double beta_ramp_fraction,
                               double beta_ramp_start, double *betas, double *gammas, double *s_sched,
                               double *scalars) {
    int peak = 0;
    for (int m = 1; m < Pts; ++m)
        if (chi[m] > chi[peak]) peak = m;
    scalars[0] = scan_s[peak];
    scalars[1] = scan_gamma[peak];
    scalars[2] = trotter_coupling(beta, scan_gamma[peak], slices);
    const double max_chi = chi[peak];
    const int degenerate = !(max_chi > 0.0) || !isfinite(max_chi);
    double floor_ = 1.0;
    if (!degenerate) {
        floor_ = chi_floor_fraction * max_chi;
        if (floor_ < 1e-12) floor_ = 1e-12;
    }
    scalars[3] = floor_;
    const double s_lo = A0 / (A0 + gamma_start), s_hi = A0 / (A0 + gamma_end);
    int n1 = 0;
    if (beta_ramp_fraction > 0.0) {
        n1 = (int)(size_t)(beta_ramp_fraction * (double)num_steps);
        if (n1 > num_steps - 2) n1 = num_steps - 2;
    }
    const int n2 = num_steps - n1;
    enum { GRID = 4096 };
    const double hs = (s_hi - s_lo) / (double)GRID;
    double *cdf = (double *)calloc(GRID + 2, sizeof(double));
#define CHI_WEIGHT(S, OUT)                                                   \
    do {                                                                    \
        const double s_ = (S);                                              \
        double c_;                                                          \
        if (s_ <= scan_s[0]) c_ = chi[0];                                   \
        else if (s_ >= scan_s[Pts - 1]) c_ = chi[Pts - 1];                  \
        else {                                                              \
            int hi_ = 1;                                                    \
            while (hi_ < Pts && scan_s[hi_] < s_) ++hi_;                    \
            const int lo_ = hi_ - 1;                                        \
            const double t_ = (s_ - scan_s[lo_]) / (scan_s[hi_] - scan_s[lo_]); \
            c_ = chi[lo_] + t_ * (chi[hi_] - chi[lo_]);                     \
        }                                                                   \
        (OUT) = c_ > floor_ ? c_ : floor_;                                  \
    } while (0)
    double w_left;
    CHI_WEIGHT(s_lo, w_left);
    for (int k = 1; k <= GRID; ++k) {
        const double sk = s_lo + (double)k * hs;
        double w_right;
        CHI_WEIGHT(sk, w_right);
        cdf[k] = cdf[k - 1] + 0.5 * (w_left + w_right) * hs;
        w_left = w_right;
    }
#undef CHI_WEIGHT
    const double cdf_end = cdf[GRID];
    for (int s = 0; s < num_steps; ++s) { betas[s] = beta; gammas[s] = gamma_start; s_sched[s] = s_lo; }
    for (int step = 0; step < n1; ++step) {
        const double frac = n1 > 1 ? (double)step / (double)(n1 - 1) : 1.0;
        betas[step] = beta_ramp_start + (beta - beta_ramp_start) * frac;
    }
    int cell = 0;
    for (int t = 0; t < n2; ++t) {
        const double target = cdf_end > 0.0 ? ((double)t / (double)(n2 - 1)) * cdf_end : 0.0;
        while (cell < GRID && cdf[cell + 1] < target) ++cell;
        const double c0 = cdf[cell], c1 = cdf[cell + 1];
        const double frac = c1 > c0 ? (target - c0) / (c1 - c0) : 0.0;
        const double s_t = s_lo + ((double)cell + frac) * hs;
        double g_t = chi_s_to_gamma(A0, s_t);
        if (g_t < gamma_end) g_t = gamma_end;
        if (g_t > gamma_start) g_t = gamma_start;
        s_sched[n1 + t] = s_t;
        gammas[n1 + t] = g_t;
    }
    free(cdf);
}

/* The pilot probe of one s point (sqa_chi_annealer.cpp:232-266): a fresh
   worldline, burn + measure parity-phase sweeps, chi_B from the pooled
   per-replica magnetisations. */
static double chi_pilot_point(const or_model *M, int P, int K, uint64_t key, int m, float B, float T4, int sweeps,
                              int burn) {
    const int n = M->n;
    ring_t R;
    ring_alloc(&R, M, P, K, key);
    ring_init(&R, DOM_PILOT_INIT | ((uint32_t)m << 8));
    const double inv_nM = 1.0 / (double)(n * P);
    double m2_sum = 0.0, mabs_sum = 0.0;
    long long count = 0;
    for (int sw = 0; sw < burn + sweeps; ++sw) {
        slice_sweep_cb(&R, (uint32_t)sw, DOM_PILOT | ((uint32_t)m << 8), B, T4, NULL);
        if (sw >= burn)
            for (int k = 0; k < K; ++k) {
                long long sum = 0;
                for (size_t i = 0; i < (size_t)P * n; ++i) sum += R.s[(size_t)k * P * n + i];
                const double mm = (double)sum * inv_nM;
                m2_sum += mm * mm;
                mabs_sum += fabs(mm);
                ++count;
            }
    }
    ring_free(&R);
    if (count < 2) return 0.0;
    const double m2_mean = m2_sum / (double)count, mabs_mean = mabs_sum / (double)count;
    const double chi = (double)(n * P) * (m2_mean - mabs_mean * mabs_mean);
    return chi > 0.0 ? chi : 0.0;
}

/* scan_chi_in != NULL replaces Stage 1 (the learned-schedule path). */
OR_EXPORT int or_chi_run(const or_model *M, int P, int K, double beta, double gamma_start, double gamma_end,
                         int num_steps, int spb, int scan_points, int scan_sweeps, int scan_burn,
                         double chi_floor_fraction, double driver_A0, double beta_ramp_fraction,
                         double beta_ramp_start, uint64_t seed, int read, const double *scan_chi_in,
                         int8_t *best_spins, double *best_E, double *trace, double *beta_sched, double *gamma_sched,
                         double *s_sched, double *scan_s, double *scan_gamma, double *scan_chi, double *scalars) {
    const int n = M->n;
    const uint64_t key = seed + (uint64_t)read;
    const double A0 = driver_A0 > 0.0 ? driver_A0 : gamma_start;
    const double s_lo = A0 / (A0 + gamma_start), s_hi = A0 / (A0 + gamma_end);
    for (int m = 0; m < scan_points; ++m) {
        const double s_m = s_lo + (s_hi - s_lo) * (double)m / (double)(scan_points - 1);
        const double g_m = chi_s_to_gamma(A0, s_m);
        scan_s[m] = s_m;
        scan_gamma[m] = g_m;
        if (scan_chi_in) {
            scan_chi[m] = scan_chi_in[m];
        } else {
            float B, T4;
            step_consts(beta, g_m, P, &B, &T4);
            scan_chi[m] = chi_pilot_point(M, P, K, key, m, B, T4, scan_sweeps, scan_burn);
        }
    }
    or_chi_schedule(scan_points, scan_s, scan_gamma, scan_chi, beta, gamma_start, gamma_end, A0, P, num_steps,
                    chi_floor_fraction, beta_ramp_fraction, beta_ramp_start, beta_sched, gamma_sched, s_sched, scalars);
    scalars[4] = A0;
    /* Stage 3: production on a fresh worldline */
    ring_t R;
    ring_alloc(&R, M, P, K, key);
    ring_init(&R, DOM_PROD_INIT);
    double *rbest = (double *)malloc(sizeof(double) * (size_t)K);
    int *rstep = (int *)malloc(sizeof(int) * (size_t)K);
    int8_t *rstate = (int8_t *)malloc((size_t)K * n);
    double *rsum = (double *)malloc(sizeof(double) * (size_t)K);
    for (int k = 0; k < K; ++k) { rbest[k] = INFINITY; rstep[k] = -1; }
    for (int step = 0; step < num_steps; ++step) {
        float B, T4;
        step_consts(beta_sched[step], gamma_sched[step], P, &B, &T4);
        for (int sw = 0; sw < spb; ++sw) slice_sweep_cb(&R, (uint32_t)(step * spb + sw), DOM_PROD, B, T4, NULL);
        for (int k = 0; k < K; ++k) {
            double sum = 0.0, emin = INFINITY;
            int tmin = 0;
            for (int t = 0; t < P; ++t) {
                double E = cell_energy(&R, k * P + t);
                sum += E;
                if (E < emin) { emin = E; tmin = t; }
            }
            rsum[k] = sum;
            if (emin < rbest[k]) {
                rbest[k] = emin; rstep[k] = step;
                memcpy(rstate + (size_t)k * n, R.s + ((size_t)k * P + tmin) * n, (size_t)n);
            }
        }
        double tot = 0.0;
        for (int k = 0; k < K; ++k) tot += rsum[k];
        trace[step] = tot / (double)(K * P);
    }
    int kb = 0;
    for (int k = 1; k < K; ++k)
        if (rbest[k] < rbest[kb] || (rbest[k] == rbest[kb] && rstep[k] < rstep[kb])) kb = k;
    *best_E = rbest[kb];
    memcpy(best_spins, rstate + (size_t)kb * n, (size_t)n);
    free(rbest); free(rstep); free(rstate); free(rsum);
    ring_free(&R);
    return 0;
}


/* ------------------------------------------------------------------ */
/* SQAAnnealer::run_optimal (sqa_annealer.cpp:499-952), one read         */
/* ------------------------------------------------------------------ */
/* Imaginary-time bond sum B = sum_{t,i} s_t,i s_t+1,i of ring k (exact). */
static long long bond_sum(const ring_t *R, int k) {
    const int n = R->n, P = R->P;
    long long b = 0;
    for (int t = 0; t < P; ++t) {
        const int8_t *a = R->s + ((size_t)k * P + t) * n, *c = R->s + ((size_t)k * P + (t + 1) % P) * n;
        for (int i = 0; i < n; ++i) b += a[i] * c[i];
    }
    return b;
}

/* chi_B = Var(B) over the step's samples of every replica
   (sqa_annealer.cpp:711-739): samples [K][ns], last_bond[K] the bond sum after
   the step (for the one-sample fallback). */
static double opt_chi_raw(const long long *samp, int K, int ns, const long long *last_bond, double nM) {
    double bs = 0.0, b2 = 0.0;
    long long total = 0;
    for (int k = 0; k < K; ++k)
        for (int j = 0; j < ns; ++j) {
            const double b = (double)samp[(size_t)k * ns + j];
            bs += b;
            b2 += b * b;
            ++total;
        }
    double var;
    if (total >= 2) {
        const double bm = bs / (double)total, b2m = b2 / (double)total;
        var = b2m - bm * bm;
    } else {
        const double ba = (double)last_bond[0] / nM;
        var = nM * (1.0 - ba * ba);
    }
    if (K == 1 && ns > 0) {
        const double ba = (double)samp[ns - 1] / nM;
        const double g = nM * (1.0 - ba * ba);
        if (g > var) var = g;
    }
    return var;
}

/* One step of sweeps at (B, T4, JP) with bond samples after every slice and
   cluster sweep; step index s drives the sweep counters. */
static void opt_sweep(ring_t *R, int s, int spb, int cls, int wls, float B, float T4, float JP, uint32_t slice_tag,
                      long long *samp) {
    const int K = R->K, ns = spb + cls;
    for (int sw = 0; sw < spb; ++sw) {
        slice_sweep(R, (uint32_t)(s * spb + sw), slice_tag, B, T4, NULL);
        for (int k = 0; k < K; ++k) samp[(size_t)k * ns + sw] = bond_sum(R, k);
    }
    for (int sw = 0; sw < cls; ++sw) {
        for (int k = 0; k < K; ++k) {
            cluster_sweep(R, k, (uint32_t)k, (uint32_t)(s * cls + sw), B, T4, JP);
            samp[(size_t)k * ns + spb + sw] = bond_sum(R, k);
        }
    }
    for (int sw = 0; sw < wls; ++sw)
        for (int k = 0; k < K; ++k) worldline_sweep(R, k, (uint32_t)k, (uint32_t)(s * wls + sw), B);
}

/* Linear interpolation of the calibration profile (sqa_annealer.cpp:832-843). */
static double opt_profile(const double *pj, const double *pc, int M, double J) {
    if (M == 0) return -1.0;
    if (J <= pj[0]) return pc[0];
    if (J >= pj[M - 1]) return pc[M - 1];
    int hi = 1;
    while (hi < M && pj[hi] < J) ++hi;
    const int lo = hi - 1;
    const double t = (J - pj[lo]) / (pj[hi] - pj[lo]);
    return pc[lo] + t * (pc[hi] - pc[lo]);
}

/* The J trajectory of a calibrated run: step t of nt sits where
   G(J) = int_{js}^{J} max(chi(J'), min_chi)^alpha dJ' (trapezoids on a 4096 grid)
   reaches t/(nt-1) of G(je) (sqa_annealer.cpp:848-872,
   sqa_parallel_tempering.cpp:768-794). */
static void opt_trajectory(const double *pj, const double *pc, int Mp, double js, double je, double min_chi,
                           double alpha, int nt, double *jt) {
    const int GRID = 4096;
    const double h = (je - js) / (double)GRID;
    double *G = (double *)calloc((size_t)GRID + 1, sizeof(double));
    double c0 = opt_profile(pj, pc, Mp, js);
    double prev = pow(c0 > min_chi ? c0 : min_chi, alpha);
    for (int k = 1; k <= GRID; ++k) {
        const double Jk = js + (double)k * h;
        const double ck = opt_profile(pj, pc, Mp, Jk);
        const double cur = pow(ck > min_chi ? ck : min_chi, alpha);
        G[k] = G[k - 1] + 0.5 * (prev + cur) * h;
        prev = cur;
    }
    const double Gt = G[GRID];
    int k = 0;
    const double den = nt > 1 ? (double)(nt - 1) : 1.0;
    for (int t = 0; t < nt; ++t) {
        const double target = Gt > 0.0 ? ((double)t / den) * Gt : 0.0;
        while (k < GRID && G[k + 1] < target) ++k;
        const double g0 = G[k], g1 = G[k + 1];
        const double fr = g1 > g0 ? (target - g0) / (g1 - g0) : 0.0;
        jt[t] = js + ((double)k + fr) * h;
    }
    free(G);
}

/* Replay form: phase-1 steps s = 0..n1-1 and phase-2 steps s = n1..num_steps-1
   use the sweep counters of step s; calibration probe m runs as step
   num_steps + m with slice tag OPTCAL (cs slice sweeps, max(cls, 1) cluster
   sweeps when cls > 0).  B = 2 beta_t / P, T4 = 4 J_perp, JP = 1 - e^{-2 J_perp}.
   scalars: calibrated eps_tilde, J_start, J_end, final J.  Returns 1 when
   run_optimal would reject its arguments. */
OR_EXPORT int or_sqa_opt_run(const or_model *M, int P, int K, double beta, double js, double je, double eps_tilde,
                             double alpha, int num_steps, int spb, int wls, int cls, int probes, int csweeps,
                             double ramp_fraction, double ramp_start, uint64_t seed, int read, int8_t *best_spins,
                             double *best_E, double *trace, double *jtrace, double *chitrace, double *scalars) {
    if (num_steps <= 0 || (spb == 0 && wls == 0 && cls == 0) || !(je > js)) return 1;
    const int n = M->n;
    const int calibrate = eps_tilde <= 0.0;
    const double nM = (double)n * (double)P;
    double min_chi = 1e-4 * nM;
    ring_t R;
    ring_alloc(&R, M, P, K, seed + (uint64_t)read);
    ring_init(&R, DOM_INIT);
    const int ns = spb + cls;
    long long *samp = (long long *)malloc(sizeof(long long) * (size_t)K * (size_t)(ns > 0 ? ns : 1) * 2 + 16);
    long long *lastb = (long long *)malloc(sizeof(long long) * (size_t)K);
    double *rbest = (double *)malloc(sizeof(double) * (size_t)K);
    int *rstep = (int *)malloc(sizeof(int) * (size_t)K);
    int8_t *rstate = (int8_t *)malloc((size_t)K * n);
    for (int k = 0; k < K; ++k) { rbest[k] = INFINITY; rstep[k] = -1; }
    const float Bc = (float)(2.0 * (beta / (double)P));
    int n1 = 0;
    if (ramp_fraction > 0.0) {
        n1 = (int)(ramp_fraction * (double)num_steps);
        if (n1 >= num_steps) n1 = num_steps - 1;
    }
    const int n2 = num_steps - n1;

#define OPT_RECORD(STEP, JV, CHIV)                                                                  \
    do {                                                                                            \
        double tot_ = 0.0;                                                                          \
        for (int k = 0; k < K; ++k) {                                                               \
            double sum_ = 0.0, emin_ = INFINITY;                                                    \
            int tmin_ = 0;                                                                          \
            for (int t = 0; t < P; ++t) {                                                           \
                const double E_ = cell_energy(&R, k * P + t);                                       \
                sum_ += E_;                                                                         \
                if (E_ < emin_) { emin_ = E_; tmin_ = t; }                                          \
            }                                                                                       \
            tot_ += sum_;                                                                           \
            if (emin_ < rbest[k]) {                                                                 \
                rbest[k] = emin_; rstep[k] = (STEP);                                                \
                memcpy(rstate + (size_t)k * n, R.s + ((size_t)k * P + tmin_) * n, (size_t)n);      \
            }                                                                                       \
        }                                                                                           \
        trace[(STEP)] = tot_ / (double)(K * P);                                                     \
        jtrace[(STEP)] = (JV);                                                                      \
        chitrace[(STEP)] = (CHIV);                                                                  \
    } while (0)

    /* phase 1: beta ramp at J_start */
    for (int s = 0; s < n1; ++s) {
        const double frac = n1 > 1 ? (double)s / (double)(n1 - 1) : 1.0;
        const double bt = ramp_start + (beta - ramp_start) * frac;
        opt_sweep(&R, s, spb, cls, wls, (float)(2.0 * (bt / (double)P)), (float)(4.0 * js),
                  (float)(1.0 - exp(-2.0 * js)), DOM_SLICE, samp);
        for (int k = 0; k < K; ++k) lastb[k] = bond_sum(&R, k);
        double chi = opt_chi_raw(samp, K, ns, lastb, nM);
        if (chi < 0.0) chi = 0.0;
        OPT_RECORD(s, js, chi);
    }
    /* calibration pre-pass */
    const int Mp = probes > 2 ? probes : 2;
    const int cs = csweeps > 1 ? csweeps : 1;
    const int pc = cls > 0 ? cls : 0;
    double *pj = (double *)malloc(sizeof(double) * (size_t)Mp), *pcv = (double *)malloc(sizeof(double) * (size_t)Mp);
    int have_profile = 0;
    const double dJ = je - js;
    if (calibrate) {
        int8_t *ss = (int8_t *)malloc((size_t)K * P * n);
        float *sg = (float *)malloc(sizeof(float) * (size_t)K * P * n);
        memcpy(ss, R.s, (size_t)K * P * n);
        memcpy(sg, R.g, sizeof(float) * (size_t)K * P * n);
        const int nsc = cs + pc;
        long long *csamp = (long long *)malloc(sizeof(long long) * (size_t)K * (size_t)nsc + 16);
        const double dJp = dJ / (double)Mp;
        double integral = 0.0, maxc = 0.0;
        for (int m = 0; m < Mp; ++m) {
            const double Jm = js + ((double)m + 0.5) * dJp;
            opt_sweep(&R, num_steps + m, cs, pc, 0, Bc, (float)(4.0 * Jm), (float)(1.0 - exp(-2.0 * Jm)), DOM_OPTCAL,
                      csamp);
            for (int k = 0; k < K; ++k) lastb[k] = bond_sum(&R, k);
            double chi = opt_chi_raw(csamp, K, nsc, lastb, nM);
            if (!(chi > 0.0)) chi = 0.0;
            pj[m] = Jm;
            pcv[m] = chi;
            integral += pow(chi > 1e-12 ? chi : 1e-12, alpha) * dJp;
            if (chi > maxc) maxc = chi;
        }
        memcpy(R.s, ss, (size_t)K * P * n);
        memcpy(R.g, sg, sizeof(float) * (size_t)K * P * n);
        free(ss); free(sg); free(csamp);
        eps_tilde = integral / (double)n2;
        if (!(eps_tilde > 0.0) || !isfinite(eps_tilde)) {
            eps_tilde = (dJ > 0.0 ? dJ : 0.0) / (double)num_steps;
            if (!(eps_tilde > 0.0)) eps_tilde = 1e-9;
        }
        min_chi = 1e-4 * maxc > 1e-12 ? 1e-4 * maxc : 1e-12;
        have_profile = 1;
    }
    scalars[0] = eps_tilde;
    scalars[1] = js;
    scalars[2] = je;
    /* the J trajectory: inverse of G(J) = int chi(J')^alpha dJ' on a 4096 grid */
    double *jt = NULL;
    if (calibrate && have_profile && je > js) {
        jt = (double *)malloc(sizeof(double) * (size_t)n2);
        opt_trajectory(pj, pcv, Mp, js, je, min_chi, alpha, n2, jt);
    }
    /* phase 2: fixed cold beta, J from the trajectory (or online) */
    double J = js;
    for (int t = 0; t < n2; ++t) {
        const int s = n1 + t;
        if (jt) J = jt[t];
        opt_sweep(&R, s, spb, cls, wls, Bc, (float)(4.0 * J), (float)(1.0 - exp(-2.0 * J)), DOM_SLICE, samp);
        for (int k = 0; k < K; ++k) lastb[k] = bond_sum(&R, k);
        const double chi_on = opt_chi_raw(samp, K, ns, lastb, nM);
        const double cp = have_profile ? opt_profile(pj, pcv, Mp, J) : -1.0;
        const double raw = cp >= 0.0 ? cp : chi_on;
        const double drive = raw > min_chi ? raw : min_chi;
        OPT_RECORD(s, J, drive);
        if (!jt) {
            const double nj = J + eps_tilde * pow(drive, -alpha);
            J = nj < je ? nj : je;
        }
    }
#undef OPT_RECORD
    scalars[3] = J;
    int kb = 0;
    for (int k = 1; k < K; ++k)
        if (rbest[k] < rbest[kb] || (rbest[k] == rbest[kb] && rstep[k] < rstep[kb])) kb = k;
    *best_E = rbest[kb];
    memcpy(best_spins, rstate + (size_t)kb * n, (size_t)n);
    free(jt); free(pj); free(pcv); free(samp); free(lastb); free(rbest); free(rstep); free(rstate);
    ring_free(&R);
    return 0;
}

/* ------------------------------------------------------------------ */
/* SQAParallelTemperingAnnealer::run_optimal                            */
/* (sqa_parallel_tempering.cpp:348-882), one read                       */
/* ------------------------------------------------------------------ */
/* One step of every rung at the shared J_perp: slice sweeps (bond sample of
   each ring after each), cluster sweeps (likewise), worldline sweeps.  Rung
   slot sl keeps its own B = 2 beta_sl / P and its random streams. */
static void ptopt_sweep(ring_t *R, const int *slot_of, const float *B, int step, int spb, int cls, int wls, float T4,
                        float JP, uint32_t slice_tag, long long *samp) {
    const int Rn = R->K, P = R->P, ns = spb + cls;
    for (int sw = 0; sw < spb; ++sw) {
        const uint32_t sigma = (uint32_t)(step * spb + sw);
        if (g_order)
            for (int k = 0; k < Rn; ++k)
                ring_slice_sweep_ref(R, k, (uint32_t)slot_of[k], sigma, slice_tag, B[slot_of[k]], T4);
        else
            for (int ph = 0; ph < 3; ++ph)
                for (int k = 0; k < Rn; ++k)
                    for (int t = 0; t < P; ++t) {
                        if (phase_of(t, P) != ph) continue;
                        const int sl = slot_of[k];
                        sweep_cell(R, k, t, (uint32_t)(sl * P + t), sigma, slice_tag, B[sl], T4);
                    }
        for (int k = 0; k < Rn; ++k) samp[(size_t)k * ns + sw] = bond_sum(R, k);
    }
    for (int sw = 0; sw < cls; ++sw)
        for (int k = 0; k < Rn; ++k) {
            const int sl = slot_of[k];
            cluster_sweep(R, k, (uint32_t)sl, (uint32_t)(step * cls + sw), B[sl], T4, JP);
            samp[(size_t)k * ns + spb + sw] = bond_sum(R, k);
        }
    for (int sw = 0; sw < wls; ++sw)
        for (int k = 0; k < Rn; ++k)
            worldline_sweep(R, k, (uint32_t)slot_of[k], (uint32_t)(step * wls + sw), B[slot_of[k]]);
}

/* Replay form: every rung runs at the one schedule J_perp of the step
   (T4 = 4 J, JP = 1 - e^{-2J}) and its own B; J starts at the hottest rung's
   coupling.  Calibration (eps_tilde <= 0) probes M points from the starting
   state, probe m as step num_steps + m with slice tag OPTCAL, then restores
   it; eps = sum_m chi_m^alpha dJ/M / num_steps and the trajectory spans all
   num_steps.  Swaps: the rung action with J_perp = 0, (beta_r/P) sum_t E_t --
   the shared Trotter terms cancel (sqa_parallel_tempering.cpp:846-861).
   P is the resolved slice count.  scalars: calibrated eps_tilde, J_start,
   resolved J_end, final J.  Returns 1 when run_optimal rejects its
   arguments. */
OR_EXPORT int or_sqapt_opt_run(const or_model *M, const double *betas, const double *gammas, int Rn, int P, int spb,
                               int wls, int cls, int steps, int swap_interval, double eps_tilde, double alpha,
                               double je, int probes, int csweeps, uint64_t seed, int read, int8_t *best_spins,
                               double *best_E, double *final_E, int8_t *final_spins, double *avg_trace,
                               double *swap_trace, double *jtrace, double *chitrace, double *scalars) {
    if (steps <= 0 || swap_interval <= 0 || (spb == 0 && wls == 0 && cls == 0) || Rn < 2) return 1;
    const int n = M->n;
    const int calibrate = eps_tilde <= 0.0;
    const double nM = (double)n * (double)P;
    const double js = trotter_coupling(betas[0], gammas[0], P);
    if (je <= 0.0) je = trotter_coupling(betas[Rn - 1], gammas[Rn - 1], P);
    if (je <= js) je = js + 1e6;
    ring_t R;
    ring_alloc(&R, M, P, Rn, seed + (uint64_t)read);
    ring_init(&R, DOM_INIT);
    int *slot_of = (int *)malloc(sizeof(int) * (size_t)Rn), *ring_in = (int *)malloc(sizeof(int) * (size_t)Rn);
    float *B = (float *)malloc(sizeof(float) * (size_t)Rn);
    double *bp = (double *)malloc(sizeof(double) * (size_t)Rn);
    double *Esum = (double *)malloc(sizeof(double) * (size_t)Rn), *Emin = (double *)malloc(sizeof(double) * (size_t)Rn);
    int *tmin = (int *)malloc(sizeof(int) * (size_t)Rn);
    long long *bond = (long long *)malloc(sizeof(long long) * (size_t)Rn);
    for (int k = 0; k < Rn; ++k) {
        slot_of[k] = ring_in[k] = k;
        B[k] = (float)(2.0 * (betas[k] / (double)P));
        bp[k] = betas[k] / (double)P;
    }
    double best = INFINITY;
    for (int k = 0; k < Rn; ++k) ring_scan(&R, k, &Esum[k], &Emin[k], &tmin[k], &bond[k]);
    for (int r = 0; r < Rn; ++r) {
        const int k = ring_in[r];
        if (Emin[k] < best) {
            best = Emin[k];
            memcpy(best_spins, R.s + ((size_t)k * P + tmin[k]) * n, (size_t)n);
        }
    }
    const int ns = spb + cls;
    const int Mp = probes > 2 ? probes : 2, cs = csweeps > 1 ? csweeps : 1, pc = cls > 0 ? cls : 0;
    const int nsc = cs + pc;
    long long *samp = (long long *)malloc(sizeof(long long) * (size_t)Rn * (size_t)(ns > nsc ? ns : nsc) + 16);
    long long lastb[1];
    double min_chi = 1e-4 * nM;
    double *pj = (double *)malloc(sizeof(double) * (size_t)Mp), *pcv = (double *)malloc(sizeof(double) * (size_t)Mp);
    double *jt = NULL;
    const double dJ = je - js;
    if (calibrate) {
        int8_t *ss = (int8_t *)malloc((size_t)Rn * P * n);
        float *sg = (float *)malloc(sizeof(float) * (size_t)Rn * P * n);
        memcpy(ss, R.s, (size_t)Rn * P * n);
        memcpy(sg, R.g, sizeof(float) * (size_t)Rn * P * n);
        const double dJp = dJ / (double)Mp;
        double integral = 0.0, maxc = 0.0;
        for (int m = 0; m < Mp; ++m) {
            const double Jm = js + ((double)m + 0.5) * dJp;
            ptopt_sweep(&R, slot_of, B, steps + m, cs, pc, 0, (float)(4.0 * Jm), (float)(1.0 - exp(-2.0 * Jm)),
                        DOM_OPTCAL, samp);
            lastb[0] = bond_sum(&R, ring_in[0]);
            double chi = opt_chi_raw(samp, Rn, nsc, lastb, nM);
            if (!(chi > 0.0)) chi = 0.0;
            pj[m] = Jm;
            pcv[m] = chi;
            integral += pow(chi > 1e-12 ? chi : 1e-12, alpha) * dJp;
            if (chi > maxc) maxc = chi;
        }
        memcpy(R.s, ss, (size_t)Rn * P * n);
        memcpy(R.g, sg, sizeof(float) * (size_t)Rn * P * n);
        free(ss); free(sg);
        eps_tilde = integral / (double)steps;
        if (!(eps_tilde > 0.0) || !isfinite(eps_tilde)) {
            eps_tilde = (dJ > 0.0 ? dJ : 0.0) / (double)steps;
            if (!(eps_tilde > 0.0)) eps_tilde = 1e-9;
        }
        min_chi = 1e-4 * maxc > 1e-12 ? 1e-4 * maxc : 1e-12;
        jt = (double *)malloc(sizeof(double) * (size_t)steps);
        opt_trajectory(pj, pcv, Mp, js, je, min_chi, alpha, steps, jt);
    }
    scalars[0] = eps_tilde;
    scalars[1] = js;
    scalars[2] = je;
    double J = js;
    for (int step = 0; step < steps; ++step) {
        if (jt) J = jt[step];
        ptopt_sweep(&R, slot_of, B, step, spb, cls, wls, (float)(4.0 * J), (float)(1.0 - exp(-2.0 * J)), DOM_SLICE,
                    samp);
        for (int k = 0; k < Rn; ++k) ring_scan(&R, k, &Esum[k], &Emin[k], &tmin[k], &bond[k]);
        for (int r = 0; r < Rn; ++r) {
            const int k = ring_in[r];
            if (Emin[k] < best) {
                best = Emin[k];
                memcpy(best_spins, R.s + ((size_t)k * P + tmin[k]) * n, (size_t)n);
            }
        }
        lastb[0] = bond[ring_in[0]];
        const double chi_on = opt_chi_raw(samp, Rn, ns, lastb, nM);
        const double cp = jt ? opt_profile(pj, pcv, Mp, J) : -1.0;
        const double raw = cp >= 0.0 ? cp : chi_on;
        const double drive = raw > min_chi ? raw : min_chi;
        jtrace[step] = J;
        chitrace[step] = drive;
        if (!jt) {
            const double nj = J + eps_tilde * pow(drive, -alpha);
            J = nj < je ? nj : je;
        }
        double acc = 0.0, att = 0.0;
        if ((step + 1) % swap_interval == 0) {
            const uint32_t w = (uint32_t)((step + 1) / swap_interval - 1);
            for (int r = 0; r + 1 < Rn; ++r) {
                const int a = ring_in[r], b = ring_in[r + 1];
                const double e_aa = bp[r] * Esum[a];
                const double e_bb = bp[r + 1] * Esum[b];
                const double e_ab = bp[r] * Esum[b];
                const double e_ba = bp[r + 1] * Esum[a];
                const double delta = (e_ab + e_ba) - (e_aa + e_bb);
                att += 1.0;
                const float u = u01(draw(R.key, (uint32_t)r, 0u, w, DOM_SWAP, 0));
                if (metropolis((float)(-delta), u)) {
                    ring_in[r] = b;
                    ring_in[r + 1] = a;
                    slot_of[b] = r;
                    slot_of[a] = r + 1;
                    acc += 1.0;
                }
            }
        }
        double avg = 0.0;
        for (int r = 0; r < Rn; ++r) avg += Emin[ring_in[r]];
        avg_trace[step] = avg / (double)Rn;
        swap_trace[step] = att > 0.0 ? acc / att : 0.0;
    }
    scalars[3] = J;
    for (int r = 0; r < Rn; ++r) {
        const int k = ring_in[r];
        final_E[r] = Emin[k];
        memcpy(final_spins + (size_t)r * n, R.s + ((size_t)k * P + tmin[k]) * n, (size_t)n);
    }
    *best_E = best;
    free(jt); free(pj); free(pcv); free(samp); free(slot_of); free(ring_in); free(B); free(bp); free(Esum);
    free(Emin); free(tmin); free(bond);
    ring_free(&R);
    return 0;
}
