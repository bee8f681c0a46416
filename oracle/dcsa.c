/*
 * dcsa.c - CPU restatement of the reference's GPU suffix-array/BWT path. TEST INFRASTRUCTURE ONLY.
 * The header dcsa.h lists, per function, the reference file:line it restates.
 * Plain sequential C (OpenMP only in the checker's independent loops), written for clarity, not speed.
 */
#define _GNU_SOURCE
#include "dcsa.h"

#include <stdlib.h>
#include <string.h>

/* ---- the cover modulo 32 (differencecover.h:29-31) -------------------------------------- */

enum { V = 32, K = 7, CLASSES = 7 };
static const int kCover[K] = {0, 1, 3, 8, 12, 19, 25};

static int is_sample_residue(int r) {
    for (int k = 0; k < K; k++) {
        if (kCover[k] == (r & (V - 1))) {
            return 1;
        }
    }
    return 0;
}

static uint8_t g_below[V], g_tie[V][V], g_class[V];
static int g_ready = 0;

static void init_tables(void) {
    if (g_ready) {
        return;
    }
    for (int r = 0; r < V; r++) {
        int below = 0;
        for (int k = 0; k < K; k++) {
            below += kCover[k] < r;
        }
        g_below[r] = (uint8_t)below;
        int d = 0;
        while (!is_sample_residue(r + d)) {
            d++;
        }
        g_class[r] = (uint8_t)d;
    }
    for (int a = 0; a < V; a++) {
        for (int b = 0; b < V; b++) {
            int k = 0;
            while (!is_sample_residue(a + k) || !is_sample_residue(b + k)) {
                k++;
            }
            g_tie[a][b] = (uint8_t)k;
        }
    }
    g_ready = 1;
}

/* differencecover.h:169-171: number of sample positions below p. */
static int64_t pack(int64_t p) {
    return (p / V) * K + g_below[p % V];
}

static int64_t sample_position(int64_t t) {
    return (t / K) * V + kCover[t % K];
}

int64_t oracle_sample_size(int64_t n) {
    init_tables();
    return n <= 0 ? 0 : pack(n);
}

void oracle_cover_tables(uint8_t below[32], uint8_t tie_offset[32 * 32], uint8_t class_of[32]) {
    init_tables();
    memcpy(below, g_below, sizeof g_below);
    memcpy(tie_offset, g_tie, sizeof g_tie);
    memcpy(class_of, g_class, sizeof g_class);
}

/* ---- suffix comparison by characters --------------------------------------------------- */

/* Compares suffixes p and q over at most limit characters; a suffix that ends first is smaller.
 * Returns <0, 0 (equal over limit characters), >0. */
static int compare_prefix(const uint8_t* text, int64_t n, int64_t p, int64_t q, int64_t limit) {
    const int64_t lp = n - p, lq = n - q;
    int64_t common = lp < lq ? lp : lq;
    if (common > limit) {
        common = limit;
    }
    const int c = memcmp(text + p, text + q, (size_t)common);
    if (c != 0) {
        return c;
    }
    if (common == limit) {
        return 0;
    }
    return lp < lq ? -1 : (lp > lq ? 1 : 0);
}

struct prefix_ctx {
    const uint8_t* text;
    int64_t n;
    int64_t limit;
};

static int cmp_positions(const void* a, const void* b, void* arg) {
    const struct prefix_ctx* c = (const struct prefix_ctx*)arg;
    const uint32_t p = *(const uint32_t*)a, q = *(const uint32_t*)b;
    const int r = compare_prefix(c->text, c->n, p, q, c->limit);
    return r != 0 ? r : (p < q ? -1 : (p > q ? 1 : 0));
}

int oracle_naive_sa(const uint8_t* text, int64_t n, uint32_t* sa) {
    if (n < 0 || n > 0xFFFFFFFFll) {
        return 1;
    }
    for (int64_t i = 0; i < n; i++) {
        sa[i] = (uint32_t)i;
    }
    struct prefix_ctx ctx = {text, n, n};
    qsort_r(sa, (size_t)n, sizeof(uint32_t), cmp_positions, &ctx);
    return 0;
}

/* ---- independent prefix doubling over all suffixes ------------------------------------- */

/* Stable counting sort of idx[0,n) by key(idx) in [0, range]. */
static void counting_sort(const uint32_t* idx, uint32_t* out, int64_t n, const uint32_t* key_of, int64_t shift,
                          int64_t total, uint32_t range, uint32_t* count) {
    memset(count, 0, ((size_t)range + 2) * sizeof(uint32_t));
    for (int64_t i = 0; i < n; i++) {
        const int64_t j = (int64_t)idx[i] + shift;
        count[(j < total ? key_of[j] : 0) + 1]++;
    }
    for (uint32_t r = 0; r <= range; r++) {
        count[r + 1] += count[r];
    }
    for (int64_t i = 0; i < n; i++) {
        const int64_t j = (int64_t)idx[i] + shift;
        out[count[j < total ? key_of[j] : 0]++] = idx[i];
    }
}

int oracle_doubling_sa(const uint8_t* text, int64_t n, uint32_t* sa) {
    if (n < 0 || n > 0xFFFFFFFEll) {
        return 1;
    }
    if (n == 0) {
        return 0;
    }
    uint32_t* rank = malloc((size_t)n * sizeof(uint32_t));
    uint32_t* next = malloc((size_t)n * sizeof(uint32_t));
    uint32_t* tmp = malloc((size_t)n * sizeof(uint32_t));
    const uint32_t range_max = (uint32_t)(n > 256 ? n : 256) + 1;
    uint32_t* count = malloc(((size_t)range_max + 2) * sizeof(uint32_t));
    if (!rank || !next || !tmp || !count) {
        free(rank), free(next), free(tmp), free(count);
        return 1;
    }
    /* Ranks start at 1, so 0 stands for "past the end", smaller than every character. */
    for (int64_t i = 0; i < n; i++) {
        rank[i] = (uint32_t)text[i] + 1;
        tmp[i] = (uint32_t)i;
    }
    counting_sort(tmp, sa, n, rank, 0, n, 257, count);
    uint32_t classes = 0;
    for (int64_t h = 1;; h *= 2) {
        /* Sort by (rank[i], rank[i+h]) with two stable passes; sa is sorted by rank[i] already. */
        counting_sort(sa, tmp, n, rank, h, n, range_max - 1, count);
        counting_sort(tmp, sa, n, rank, 0, n, range_max - 1, count);
        classes = 0;
        for (int64_t k = 0; k < n; k++) {
            const uint32_t i = sa[k];
            if (k == 0) {
                classes = 1;
            } else {
                const uint32_t j = sa[k - 1];
                const uint32_t a2 = (int64_t)i + h < n ? rank[i + h] : 0;
                const uint32_t b2 = (int64_t)j + h < n ? rank[j + h] : 0;
                if (rank[i] != rank[j] || a2 != b2) {
                    classes++;
                }
            }
            next[i] = classes;
        }
        memcpy(rank, next, (size_t)n * sizeof(uint32_t));
        if ((int64_t)classes == n) {
            break;
        }
    }
    free(rank), free(next), free(tmp), free(count);
    return 0;
}

/* ---- step 2: sample ranks (samplerank.cuh:1-20) ------------------------------------------ */

struct group_ctx {
    const uint32_t* group;   /* group id per compact sample index */
    int64_t n, h;
};

/* Key of sample position p in a doubling round: (group of p, 1 + group of p+h, or 0 past the end). */
static int cmp_doubling(const void* a, const void* b, void* arg) {
    const struct group_ctx* c = (const struct group_ctx*)arg;
    const uint32_t p = *(const uint32_t*)a, q = *(const uint32_t*)b;
    const uint32_t gp = c->group[pack(p)], gq = c->group[pack(q)];
    if (gp != gq) {
        return gp < gq ? -1 : 1;
    }
    const uint64_t sp = (int64_t)p + c->h < c->n ? (uint64_t)c->group[pack(p + c->h)] + 1 : 0;
    const uint64_t sq = (int64_t)q + c->h < c->n ? (uint64_t)c->group[pack(q + c->h)] + 1 : 0;
    if (sp != sq) {
        return sp < sq ? -1 : 1;
    }
    return p < q ? -1 : (p > q ? 1 : 0);
}

int oracle_dc_sample_ranks(const uint8_t* text, int64_t n, uint32_t* ranks) {
    init_tables();
    if (n < 0 || n > 0xFFFFFFFEll) {
        return 1;
    }
    const int64_t m = oracle_sample_size(n);
    if (m == 0) {
        return 0;
    }
    uint32_t* order = malloc((size_t)m * sizeof(uint32_t));
    uint32_t* fresh = malloc((size_t)m * sizeof(uint32_t));
    if (!order || !fresh) {
        free(order), free(fresh);
        return 1;
    }
    for (int64_t t = 0; t < m; t++) {
        order[t] = (uint32_t)sample_position(t);
    }
    /* Groups of the first V characters (shorter first when one ends inside the window). */
    struct prefix_ctx pctx = {text, n, V};
    qsort_r(order, (size_t)m, sizeof(uint32_t), cmp_positions, &pctx);
    int64_t head = 0;
    for (int64_t k = 0; k < m; k++) {
        if (k > 0 && compare_prefix(text, n, order[k - 1], order[k], V) != 0) {
            head = k;
        }
        ranks[pack(order[k])] = (uint32_t)head;
    }
    /* Doubling: groups sharing h characters (h a multiple of V) are split by the group at p + h. */
    for (int64_t h = V;; h *= 2) {
        int singletons = 1;
        for (int64_t k = 1; k < m && singletons; k++) {
            singletons = ranks[pack(order[k - 1])] != ranks[pack(order[k])];
        }
        if (singletons) {
            break;
        }
        struct group_ctx gctx = {ranks, n, h};
        qsort_r(order, (size_t)m, sizeof(uint32_t), cmp_doubling, &gctx);
        /* All keys read from the previous round's ids before any is rewritten. */
        head = 0;
        for (int64_t k = 0; k < m; k++) {
            if (k > 0) {
                const uint32_t p = order[k - 1], q = order[k];
                const uint32_t gp = ranks[pack(p)], gq = ranks[pack(q)];
                const uint64_t sp = (int64_t)p + h < n ? (uint64_t)ranks[pack(p + h)] + 1 : 0;
                const uint64_t sq = (int64_t)q + h < n ? (uint64_t)ranks[pack(q + h)] + 1 : 0;
                if (gp != gq || sp != sq) {
                    head = k;
                }
            }
            fresh[k] = (uint32_t)head;
        }
        for (int64_t k = 0; k < m; k++) {
            ranks[pack(order[k])] = fresh[k];
        }
        if (h > n) {
            break;
        }
    }
    free(order), free(fresh);
    return 0;
}

/* ---- step 3: class lists (classsort.cuh:1-20,100-123) ------------------------------------ */

static void class_starts(int64_t n, int64_t* start) {
    init_tables();
    int64_t size[CLASSES] = {0};
    for (int r = 0; r < V; r++) {
        size[g_class[r]] += n / V + (r < n % V ? 1 : 0);
    }
    start[0] = 0;
    for (int d = 0; d < CLASSES; d++) {
        start[d + 1] = start[d] + size[d];
    }
}

int oracle_dc_class_lists(const uint8_t* text, int64_t n, const uint32_t* ranks, uint32_t* lists, int64_t* start) {
    init_tables();
    if (n < 0 || n > 0xFFFFFFFEll) {
        return 1;
    }
    class_starts(n, start);
    const int64_t m = start[1];
    for (int64_t t = 0; t < m; t++) {
        lists[ranks[t]] = (uint32_t)sample_position(t);
    }
    uint32_t* emitted = malloc(((size_t)(start[CLASSES] - start[0]) + 1) * sizeof(uint32_t));
    if (!emitted) {
        return 1;
    }
    for (int d = 1; d < CLASSES; d++) {
        const uint32_t* previous = lists + start[d - 1];
        const int64_t count = start[d] - start[d - 1];
        int64_t e = 0;
        /* Walk class d-1 with n (the empty suffix, smallest) prepended; keep predecessors in class d. */
        for (int64_t k = 0; k <= count; k++) {
            const int64_t p = k == 0 ? n : previous[k - 1];
            if (p > 0 && g_class[(p - 1) % V] == d) {
                emitted[e++] = (uint32_t)(p - 1);
            }
        }
        if (e != start[d + 1] - start[d]) {
            free(emitted);
            return 2;
        }
        /* Stable by the first character. */
        int64_t bucket[257] = {0};
        for (int64_t k = 0; k < e; k++) {
            bucket[text[emitted[k]] + 1]++;
        }
        for (int c = 0; c < 256; c++) {
            bucket[c + 1] += bucket[c];
        }
        uint32_t* out = lists + start[d];
        for (int64_t k = 0; k < e; k++) {
            out[bucket[text[emitted[k]]]++] = emitted[k];
        }
    }
    free(emitted);
    return 0;
}

/* ---- step 4: merge by the difference-cover comparison (merge.cuh:53-71) ------------------ */

static int dc_less(const uint8_t* text, int64_t n, const uint32_t* ranks, int64_t i, int64_t j) {
    const int64_t k = g_tie[i % V][j % V];
    int64_t common = k;
    if (n - i < common) {
        common = n - i;
    }
    if (n - j < common) {
        common = n - j;
    }
    const int c = memcmp(text + i, text + j, (size_t)common);
    if (c != 0) {
        return c < 0;
    }
    if (common < k || i + k == n || j + k == n) {
        return i > j; /* one is a prefix of the other: the shorter is smaller */
    }
    return ranks[pack(i + k)] < ranks[pack(j + k)];
}

int oracle_dc_merge(const uint8_t* text, int64_t n, const uint32_t* ranks, const uint32_t* lists,
                    const int64_t* start, uint32_t* sa) {
    init_tables();
    int64_t head[CLASSES];
    for (int d = 0; d < CLASSES; d++) {
        head[d] = start[d];
    }
    for (int64_t r = 0; r < n; r++) {
        int best = -1;
        for (int d = 0; d < CLASSES; d++) {
            if (head[d] == start[d + 1]) {
                continue;
            }
            if (best < 0 || dc_less(text, n, ranks, lists[head[d]], lists[head[best]])) {
                best = d;
            }
        }
        if (best < 0) {
            return 2;
        }
        sa[r] = lists[head[best]++];
    }
    return 0;
}

int oracle_dc_sa(const uint8_t* text, int64_t n, uint32_t* sa) {
    init_tables();
    if (n < 0 || n > 0xFFFFFFFEll) {
        return 1;
    }
    if (n == 0) {
        return 0;
    }
    const int64_t m = oracle_sample_size(n);
    uint32_t* ranks = malloc(((size_t)m + 1) * sizeof(uint32_t));
    uint32_t* lists = malloc((size_t)n * sizeof(uint32_t));
    int64_t start[CLASSES + 1];
    int status = (!ranks || !lists) ? 1 : 0;
    if (!status) {
        status = oracle_dc_sample_ranks(text, n, ranks);
    }
    if (!status) {
        status = oracle_dc_class_lists(text, n, ranks, lists, start);
    }
    if (!status) {
        status = oracle_dc_merge(text, n, ranks, lists, start, sa);
    }
    free(ranks), free(lists);
    return status;
}

/* ---- derived outputs ------------------------------------------------------------------- */

void oracle_sample_ranks_from_sa(const uint32_t* sa, int64_t n, uint32_t* ranks) {
    init_tables();
    uint32_t rank = 0;
    for (int64_t i = 0; i < n; i++) {
        if (is_sample_residue((int)(sa[i] % V))) {
            ranks[pack(sa[i])] = rank++;
        }
    }
}

int64_t oracle_bwt_from_sa(const uint8_t* text, int64_t n, const uint32_t* sa, uint8_t* bwt) {
    if (n <= 0) {
        return 0;
    }
    int64_t primary = 0, out = 0;
    bwt[out++] = text[n - 1]; /* the sentinel's row */
    for (int64_t row = 0; row < n; row++) {
        if (sa[row] == 0) {
            primary = row + 1;
        } else {
            bwt[out++] = text[sa[row] - 1];
        }
    }
    return primary;
}

/* ---- checkers (checker.cpp:53-109, 196-245), 64-bit ------------------------------------- */

int oracle_check_sa(const uint8_t* text, int64_t n, const uint32_t* sa, int64_t* index) {
    if (index) {
        *index = -1;
    }
    if (n <= 0) {
        return 1;
    }
    uint32_t* isa = malloc((size_t)n * sizeof(uint32_t));
    if (!isa) {
        return 0;
    }
    int64_t first = INT64_MAX;
#pragma omp parallel for reduction(min : first)
    for (int64_t i = 0; i < n; i++) {
        if ((int64_t)sa[i] >= n) {
            first = i < first ? i : first;
        } else {
            isa[sa[i]] = (uint32_t)i;
        }
    }
    if (first == INT64_MAX) {
        /* Of two equal entries, only one owns the inverse slot. */
#pragma omp parallel for reduction(min : first)
        for (int64_t i = 0; i < n; i++) {
            if (isa[sa[i]] != (uint32_t)i) {
                first = i < first ? i : first;
            }
        }
    }
    if (first == INT64_MAX) {
#pragma omp parallel for reduction(min : first)
        for (int64_t i = 0; i < n - 1; i++) {
            const int64_t l = sa[i], r = sa[i + 1];
            int ok = text[l] < text[r];
            if (text[l] == text[r]) {
                const int64_t ln = l + 1 < n ? (int64_t)isa[l + 1] : -1;
                const int64_t rn = r + 1 < n ? (int64_t)isa[r + 1] : -1;
                ok = ln < rn;
            }
            if (!ok) {
                first = i < first ? i : first;
            }
        }
    }
    free(isa);
    if (first != INT64_MAX) {
        if (index) {
            *index = first;
        }
        return 0;
    }
    return 1;
}

int oracle_check_bwt(const uint8_t* text, int64_t n, const uint8_t* bwt, int64_t primary, int64_t* index) {
    if (index) {
        *index = -1;
    }
    if (n == 0) {
        return primary == 0;
    }
    if (primary < 1 || primary > n) {
        return 0;
    }
    uint32_t* lf = malloc((size_t)n * sizeof(uint32_t));
    if (!lf) {
        return 0;
    }
    int64_t next[256] = {0};
    for (int64_t u = 0; u < n; u++) {
        next[bwt[u]]++;
    }
    for (int64_t c = 0, sum = 1; c < 256; c++) {
        const int64_t count = next[c];
        next[c] = sum;
        sum += count;
    }
    for (int64_t u = 0; u < n; u++) {
        lf[u] = (uint32_t)next[bwt[u]]++;
    }
    int64_t row = 0;
    for (int64_t i = n - 1; i >= 0; i--) {
        if (row == primary) {
            if (index) {
                *index = i;
            }
            free(lf);
            return 0;
        }
        const int64_t u = row < primary ? row : row - 1;
        if (bwt[u] != text[i]) {
            if (index) {
                *index = i;
            }
            free(lf);
            return 0;
        }
        row = lf[u];
    }
    free(lf);
    if (row != primary) {
        if (index) {
            *index = 0;
        }
        return 0;
    }
    return 1;
}

/* ---- LCP array (no counterpart in the reference) ---------------------------------------- */

int oracle_lcp(const uint8_t* text, int64_t n, const uint32_t* sa, uint32_t* lcp) {
    if (n <= 0) {
        return 1;
    }
    /* phi[p] = the suffix just before suffix p in suffix order (n for the smallest suffix); then
     * plcp[p] = lcp(p, phi[p]) in text order, where plcp[p + 1] >= plcp[p] - 1 lets the common
     * length carry from one position to the next (linear total work). */
    uint32_t* phi = malloc((size_t)n * sizeof(uint32_t));
    if (!phi) {
        return 0;
    }
    phi[sa[0]] = (uint32_t)n;
    for (int64_t r = 1; r < n; r++) {
        phi[sa[r]] = sa[r - 1];
    }
    int64_t h = 0;
    for (int64_t p = 0; p < n; p++) {
        const int64_t q = phi[p];
        if (q == n) {
            h = 0;
            phi[p] = 0;
            continue;
        }
        while (p + h < n && q + h < n && text[p + h] == text[q + h]) {
            h++;
        }
        phi[p] = (uint32_t)h; /* phi[p] is not read again: it becomes plcp[p] */
        if (h > 0) {
            h--;
        }
    }
    for (int64_t r = 0; r < n; r++) {
        lcp[r] = phi[sa[r]];
    }
    free(phi);
    return 1;
}
