/*
 * paswas_oracle.c -- CPU restatement of the pyPaSWAS Smith-Waterman hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle the CUDA engine is checked
 * against; it is linked only by tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py.  The shipped engine never calls it.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks this file against golden
 * fixtures produced by the reference's own code (its CUDA kernels compiled for
 * the CPU plus its unmodified Python host walk, tests/golden/make_golden.py).
 *
 * It restates, literally and in the reference's own order:
 *   - calculateScore            pyPaSWAS/Core/cuda/default_main.cu:130-303
 *   - calculateScoreAffineGap   pyPaSWAS/Core/cuda/default_main.cu:317-561
 *   - traceback                 pyPaSWAS/Core/cuda/default_main.cu:566-714
 *   - tracebackAffineGap (+ tracebackStep*)  default_main.cu:716-909
 *   - the block anti-diagonal launch loops   pyPaSWAS/Core/SmithWaterman.py:592-655
 *   - the host walk _print_alignments         pyPaSWAS/Core/SmithWaterman.py:665-841
 * using full fp32 matrices per pair and the sign-bit marking of the reference.
 *
 * Pinned choices where the reference is nondeterministic:
 *   - starting points are emitted in the order of a sequential execution of the
 *     traceback launches: block anti-diagonal descending, blocks in CUDA linear
 *     block order (k = blockIdx.y / NUMBER_TARGETS ascending, i.e. block x
 *     descending; then target; then query), cell anti-diagonal descending inside
 *     the block, then linear thread index (threadIdx.x fastest) ascending;
 *   - the zero-copy direction buffer starts zeroed for every pair.
 * Pairs are computed on their own 8-padded shape; with non-positive gap
 * penalties padded cells cannot change any result (they only feed the block
 * maximum, and their scores never exceed their real neighbours').
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define SHARED 8
#define FILL_SCORE (-1E10f)        /* default_main.cu:19 */
#define AFFINE_GAP_INIT (-1E10f)   /* default_main.cu:29 */
#define NO_DIRECTION 32            /* pyPaSWAS/Core/__init__.py:7-13 */
#define UPPER_LEFT 1
#define UPPER 2
#define LEFT 3
#define STOP_DIRECTION 64
#define IN_ALIGNMENT 96
#define MAIN_MATRIX (UPPER_LEFT << 2) /* default_direction.cu:9-18 */
#define I_MATRIX (UPPER << 2)
#define J_MATRIX (LEFT << 2)
#define DIRECTION_MASK 3
#define MATRIX_MASK 12

typedef struct {
    int dim;              /* scoring matrix dimension (26 for DNA-RNA / BLOSUM) */
    int char_offset;      /* characterOffset of the score (Scores.py) */
    const float* matrix;  /* dim*dim, row = query char, col = target char */
    float gap;            /* gapScore */
    float ext;            /* gapExtension (only used when affine) */
    int affine;           /* gap_extension != None (SmithWaterman.py:149) */
    float lower_limit;    /* LOWER_LIMIT_SCORE as compiled (fp32) */
    float minimum_score;  /* MINIMUM_SCORE as compiled (fp32) */
} orc_params;

/* StartingPoint struct of default_main.cu:66-76 / StartingPoint.py:7-17. */
typedef struct {
    uint32_t sequence, target, block_x, block_y, value_x, value_y;
    float score, max_score, pos_score;
} orc_start;

typedef struct {
    int32_t query, target;          /* indices into the query / target lists */
    int32_t s_start, s_end, t_start, t_end;
    float score;
    int32_t matches, mismatches;
    int32_t n_cols;                 /* length of the three alignment strings */
    int64_t str_offset;             /* into the string buffer: seq | align | target */
} orc_hit;

static inline float sign_mark(float v) {
    uint32_t u;
    memcpy(&u, &v, 4);
    u |= 0x80000000u;
    memcpy(&v, &u, 4);
    return v;
}

static inline float inner_score(const orc_params* p, uint8_t a, uint8_t b) {
    /* default_main.cu:234 -- FILL character gives FILL_SCORE */
    if (a == 0 || b == 0) return FILL_SCORE;
    return p->matrix[(a - p->char_offset) * p->dim + (b - p->char_offset)];
}

typedef struct {
    int X, Y;           /* padded shape, multiples of 8 */
    float* H;           /* M matrix  [X][Y] */
    float* I;           /* I matrix  [X][Y] (affine) */
    float* J;           /* J matrix  [X][Y] (affine) */
    uint8_t* dir;       /* device direction matrix [X][Y] */
    uint8_t* zc;        /* zero-copy direction buffer [X][Y] */
    float max;          /* pair maximum (last block of the maxima chain) */
} pair_mats;

#define AT(m, x, y) ((m)[(size_t)(x) * P->Y + (y)])

/* Score fill of one pair; cell order is irrelevant to the values, only the
 * dependency (x-1, y-1), (x-1, y), (x, y-1) matters. */
static void score_linear(const orc_params* p, pair_mats* P, const uint8_t* q, const uint8_t* t) {
    float mx = 0.0f;
    for (int x = 0; x < P->X; ++x) {
        for (int y = 0; y < P->Y; ++y) {
            float inner = inner_score(p, q[x], t[y]);
            float hd = (x && y) ? AT(P->H, x - 1, y - 1) : 0.0f;
            float hl = x ? AT(P->H, x - 1, y) : 0.0f;
            float hu = y ? AT(P->H, x, y - 1) : 0.0f;
            /* default_main.cu:255-271 */
            float ulS = hd + inner, lS = hl + p->gap, uS = hu + p->gap;
            float cur = 0.0f;
            uint8_t d = NO_DIRECTION;
            if (cur < lS) { cur = lS; d = LEFT; }
            if (cur < uS) { cur = uS; d = UPPER; }
            if (cur < ulS) { cur = ulS; d = UPPER_LEFT; }
            AT(P->H, x, y) = inner == FILL_SCORE ? 0.0f : cur;
            AT(P->dir, x, y) = d;
            /* block maxima chain (:169-180,274-288,297-298) == max of every
             * cell's currentScore */
            mx = fmaxf(mx, cur);
        }
    }
    P->max = mx;
}

static void score_affine(const orc_params* p, pair_mats* P, const uint8_t* q, const uint8_t* t) {
    float mx = 0.0f;
    const float ge = p->gap + p->ext; /* gapScore + gapExtension, folded (:487,502) */
    for (int x = 0; x < P->X; ++x) {
        for (int y = 0; y < P->Y; ++y) {
            float inner = inner_score(p, q[x], t[y]);
            float md = (x && y) ? AT(P->H, x - 1, y - 1) : 0.0f;
            float id = (x && y) ? AT(P->I, x - 1, y - 1) : AFFINE_GAP_INIT;
            float jd = (x && y) ? AT(P->J, x - 1, y - 1) : AFFINE_GAP_INIT;
            float mu = y ? AT(P->H, x, y - 1) : 0.0f;
            float iu = y ? AT(P->I, x, y - 1) : AFFINE_GAP_INIT;
            float ml = x ? AT(P->H, x - 1, y) : 0.0f;
            float jl = x ? AT(P->J, x - 1, y) : AFFINE_GAP_INIT;
            /* default_main.cu:467-483 */
            float m_M = md + inner, m_I = id + inner, m_J = jd + inner;
            float cur = 0.0f;
            uint8_t d = NO_DIRECTION, di = NO_DIRECTION, dj = NO_DIRECTION;
            if (cur < m_I) { cur = m_I; d = UPPER_LEFT | MAIN_MATRIX; }
            if (cur < m_J) { cur = m_J; d = UPPER_LEFT | MAIN_MATRIX; }
            if (cur < m_M) { cur = m_M; d = UPPER_LEFT | MAIN_MATRIX; }
            float mstore = inner == FILL_SCORE ? 0.0f : cur;
            /* I matrix :486-498 */
            float ci = AFFINE_GAP_INIT;
            float a = ge + mu, b = p->ext + iu;
            if (ci < b) { ci = b; di = UPPER | I_MATRIX; }
            if (ci < a) { ci = a; di = UPPER | I_MATRIX; }
            float istore = ci < 0 ? AFFINE_GAP_INIT : ci;
            /* J matrix :501-513 */
            float cj = AFFINE_GAP_INIT;
            a = ge + ml;
            b = p->ext + jl;
            if (cj < b) { cj = b; dj = LEFT | J_MATRIX; }
            if (cj < a) { cj = a; dj = LEFT | J_MATRIX; }
            float jstore = cj < 0 ? AFFINE_GAP_INIT : cj;
            /* best source :515-526 */
            cur = fmaxf(cur, fmaxf(ci, cj));
            if (cur > 0) {
                if (cur == mstore) {
                } else if (cur == istore) {
                    d = di;
                } else if (cur == jstore) {
                    d = dj;
                }
            }
            AT(P->H, x, y) = mstore;
            AT(P->I, x, y) = istore;
            AT(P->J, x, y) = jstore;
            AT(P->dir, x, y) = d;
            mx = fmaxf(mx, cur);
        }
    }
    P->max = mx;
}

/* Emission key of a starting point, see the header comment. */
typedef struct {
    float score;
    int32_t neg_diag, neg_bx, target, query, neg_i, ty;
    int32_t src; /* index into the start array */
} start_key;

typedef struct {
    orc_start* starts;
    start_key* keys;
    int n, cap;
} start_sink;

static void emit_start(start_sink* s, const orc_start* st) {
    if (s->n < s->cap) {
        s->starts[s->n] = *st;
        start_key* k = &s->keys[s->n];
        int x = st->block_x * SHARED + st->value_x, y = st->block_y * SHARED + st->value_y;
        (void)x;
        (void)y;
        k->score = st->score;
        k->neg_diag = -(int32_t)(st->block_x + st->block_y);
        k->neg_bx = -(int32_t)st->block_x;
        k->target = (int32_t)st->target;
        k->query = (int32_t)st->sequence;
        k->neg_i = -(int32_t)(st->value_x + st->value_y);
        k->ty = (int32_t)st->value_y;
        k->src = s->n;
    }
    s->n++;
}

/* One block of the linear traceback kernel (default_main.cu:596-713). */
static void traceback_block_linear(const orc_params* p, pair_mats* P, int bx, int by, float pos, uint32_t qi,
                                   uint32_t ti, start_sink* sink) {
    uint8_t dir[SHARED][SHARED];
    for (int tx = 0; tx < SHARED; ++tx)
        for (int ty = 0; ty < SHARED; ++ty) dir[tx][ty] = AT(P->dir, bx * SHARED + tx, by * SHARED + ty);
    for (int i = 2 * SHARED - 1; i >= 0; --i) {
        /* phase: starting points (:609-627), threads in linear order */
        for (int ty = 0; ty < SHARED; ++ty) {
            int tx = i - ty;
            if (tx < 0 || tx >= SHARED) continue;
            int x = bx * SHARED + tx, y = by * SHARED + ty;
            float v = AT(P->H, x, y);
            if (dir[tx][ty] == UPPER_LEFT && v >= p->lower_limit * P->max && v >= pos) {
                orc_start st = {qi, ti, (uint32_t)bx, (uint32_t)by, (uint32_t)tx, (uint32_t)ty, v, P->max, pos};
                emit_start(sink, &st);
                AT(P->H, x, y) = sign_mark(v);
            }
        }
        /* UL / UP / LEFT propagation phases (:631-700) */
        for (int phase = 0; phase < 3; ++phase) {
            for (int ty = 0; ty < SHARED; ++ty) {
                int tx = i - ty;
                if (tx < 0 || tx >= SHARED) continue;
                int x = bx * SHARED + tx, y = by * SHARED + ty;
                if (!(AT(P->H, x, y) < 0)) continue;
                int want = phase == 0 ? UPPER_LEFT : (phase == 1 ? UPPER : LEFT);
                if (dir[tx][ty] != want) continue;
                int px = x - (want == UPPER ? 0 : 1), py = y - (want == LEFT ? 0 : 1);
                if (px < 0 || py < 0) continue; /* matrix edge: nothing happens */
                float value = AT(P->H, px, py);
                if (value == 0.0f)
                    dir[tx][ty] = STOP_DIRECTION;
                else
                    AT(P->H, px, py) = sign_mark(value);
            }
        }
    }
    /* write-back of marked cells to the zero-copy buffer (:707-710) */
    for (int tx = 0; tx < SHARED; ++tx)
        for (int ty = 0; ty < SHARED; ++ty) {
            int x = bx * SHARED + tx, y = by * SHARED + ty;
            if (AT(P->H, x, y) < 0) AT(P->zc, x, y) = dir[tx][ty];
        }
}

/* One block of the affine traceback kernel (default_main.cu:836-908). */
static void traceback_block_affine(const orc_params* p, pair_mats* P, int bx, int by, float pos, uint32_t qi,
                                   uint32_t ti, start_sink* sink) {
    uint8_t dir[SHARED][SHARED], src[SHARED][SHARED];
    for (int tx = 0; tx < SHARED; ++tx)
        for (int ty = 0; ty < SHARED; ++ty) {
            uint8_t d = AT(P->dir, bx * SHARED + tx, by * SHARED + ty);
            dir[tx][ty] = d & DIRECTION_MASK;
            src[tx][ty] = d & MATRIX_MASK;
        }
    for (int i = 2 * SHARED - 1; i >= 0; --i) {
        for (int ty = 0; ty < SHARED; ++ty) {
            int tx = i - ty;
            if (tx < 0 || tx >= SHARED) continue;
            int x = bx * SHARED + tx, y = by * SHARED + ty;
            float v = AT(P->H, x, y);
            if (src[tx][ty] == MAIN_MATRIX && v >= p->lower_limit * P->max && v >= pos) {
                orc_start st = {qi, ti, (uint32_t)bx, (uint32_t)by, (uint32_t)tx, (uint32_t)ty, v, P->max, pos};
                emit_start(sink, &st);
                AT(P->H, x, y) = sign_mark(v);
            }
        }
        for (int ty = 0; ty < SHARED; ++ty) {
            int tx = i - ty;
            if (tx < 0 || tx >= SHARED) continue;
            int x = bx * SHARED + tx, y = by * SHARED + ty;
            float m = AT(P->H, x, y), iv = AT(P->I, x, y), jv = AT(P->J, x, y);
            int go = (m < 0 && src[tx][ty] == MAIN_MATRIX) ||
                     (iv < 0 && iv > AFFINE_GAP_INIT && src[tx][ty] == I_MATRIX) ||
                     (jv < 0 && jv > AFFINE_GAP_INIT && src[tx][ty] == J_MATRIX);
            if (!go) continue;
            if (dir[tx][ty] == UPPER_LEFT) { /* tracebackStepLeftUp :716-754 */
                if (x > 0 && y > 0) {
                    float value = AT(P->H, x - 1, y - 1);
                    if (value == 0.0f)
                        dir[tx][ty] = STOP_DIRECTION;
                    else
                        AT(P->H, x - 1, y - 1) = sign_mark(value);
                }
            } else if (dir[tx][ty] == UPPER) { /* tracebackStepUp :756-776 */
                if (y > 0) AT(P->I, x, y - 1) = sign_mark(AT(P->I, x, y - 1));
            } else if (dir[tx][ty] == LEFT) { /* tracebackStepLeft :778-800 */
                if (x > 0) AT(P->J, x - 1, y) = sign_mark(AT(P->J, x - 1, y));
            }
        }
    }
    for (int tx = 0; tx < SHARED; ++tx)
        for (int ty = 0; ty < SHARED; ++ty)
            if (src[tx][ty]) AT(P->zc, bx * SHARED + tx, by * SHARED + ty) = dir[tx][ty];
}

/* Reverse block anti-diagonal sweep of SmithWaterman._traceback_host
 * (SmithWaterman.py:626-655); within a launch blocks go in CUDA linear order,
 * i.e. k = blockIdx.y / NUMBER_TARGETS ascending, which is block x descending. */
static void traceback_pair(const orc_params* p, pair_mats* P, float pos, uint32_t qi, uint32_t ti,
                           start_sink* sink) {
    if (!(P->max >= p->minimum_score)) return; /* :596 */
    const int XB = P->X / SHARED, YB = P->Y / SHARED;
    for (int d = XB + YB - 2; d >= 0; --d) {
        int bx_hi = d < XB - 1 ? d : XB - 1;
        int bx_lo = d - (YB - 1) > 0 ? d - (YB - 1) : 0;
        for (int bx = bx_hi; bx >= bx_lo; --bx) {
            int by = d - bx;
            if (p->affine)
                traceback_block_affine(p, P, bx, by, pos, qi, ti, sink);
            else
                traceback_block_linear(p, P, bx, by, pos, qi, ti, sink);
        }
    }
}

/* emission order alone (the order of the reference's starting-point buffer) */
static int emit_cmp(const void* a, const void* b) {
    const start_key* x = (const start_key*)a;
    const start_key* y = (const start_key*)b;
#define CMPF(f) if (x->f != y->f) return x->f < y->f ? -1 : 1
    CMPF(neg_diag);
    CMPF(neg_bx);
    CMPF(target);
    CMPF(query);
    CMPF(neg_i);
    CMPF(ty);
    CMPF(src);
#undef CMPF
    return 0;
}

static int key_cmp(const void* a, const void* b) {
    const start_key* x = (const start_key*)a;
    const start_key* y = (const start_key*)b;
    if (x->score != y->score) return x->score < y->score ? -1 : 1;
#define CMPF(f) if (x->f != y->f) return x->f < y->f ? -1 : 1
    CMPF(neg_diag);
    CMPF(neg_bx);
    CMPF(target);
    CMPF(query);
    CMPF(neg_i);
    CMPF(ty);
    CMPF(src);
#undef CMPF
    return 0;
}

/*
 * Runs the whole path for all (query, target) pairs: score fill, traceback
 * sweep, and the host walk of SmithWaterman._print_alignments.
 *
 * Sequences are passed unpadded and already upper-cased (SWSeq.extentToFillGPU).
 * pos_score is indexed [target * nq + query] like maxPossibleScore
 * (SmithWatermanCuda.py:269-275).  id_key: records whose id strings are equal
 * carry equal keys (same-id hits are skipped, SmithWaterman.py:752-755).
 * start_cap: how many starting points the walk may use (100 per pair in the
 * reference, SmithWaterman.py:683-685); < 0 means unlimited.
 * Outputs: pair_max [query * nt + target]; hits in walk order; strings for hit
 * h at strbuf + str_offset: sequence_match, alignment, target_match, each
 * n_cols bytes.  Returns 0, or -1 when a capacity was exceeded (n_* tell the
 * required sizes).
 */
int orc_run(const orc_params* p, int nq, const uint8_t* q_res, const int64_t* q_off, int nt,
            const uint8_t* t_res, const int64_t* t_off, const int32_t* q_idkey, const int32_t* t_idkey,
            const float* pos_score, double host_min_score, int64_t start_cap, float* pair_max,
            orc_start* starts_out, int64_t max_starts, int64_t* n_starts, orc_hit* hits, int64_t max_hits,
            int64_t* n_hits, char* strbuf, int64_t strbuf_cap, int64_t* str_used) {
    int64_t cap = 1 << 16;
    start_sink sink;
    sink.cap = (int)cap;
    sink.n = 0;
    sink.starts = (orc_start*)malloc(sizeof(orc_start) * cap);
    sink.keys = (start_key*)malloc(sizeof(start_key) * cap);
    int rc = 0;

    /* keep every pair's zero-copy buffer for the walk */
    uint8_t** zc = (uint8_t**)calloc((size_t)nq * nt, sizeof(uint8_t*));
    int* zX = (int*)calloc((size_t)nq * nt, sizeof(int));
    int* zY = (int*)calloc((size_t)nq * nt, sizeof(int));

    for (int ti = 0; ti < nt; ++ti) {
        for (int qi = 0; qi < nq; ++qi) {
            int lq = (int)(q_off[qi + 1] - q_off[qi]), lt = (int)(t_off[ti + 1] - t_off[ti]);
            pair_mats P;
            P.X = (lq + SHARED - 1) / SHARED * SHARED;
            P.Y = (lt + SHARED - 1) / SHARED * SHARED;
            if (P.X == 0) P.X = SHARED;
            if (P.Y == 0) P.Y = SHARED;
            size_t cells = (size_t)P.X * P.Y;
            uint8_t* qp = (uint8_t*)calloc(P.X, 1);
            uint8_t* tp = (uint8_t*)calloc(P.Y, 1);
            memcpy(qp, q_res + q_off[qi], lq);
            memcpy(tp, t_res + t_off[ti], lt);
            P.H = (float*)calloc(cells, 4);
            P.I = p->affine ? (float*)calloc(cells, 4) : NULL;
            P.J = p->affine ? (float*)calloc(cells, 4) : NULL;
            P.dir = (uint8_t*)calloc(cells, 1);
            P.zc = (uint8_t*)calloc(cells, 1);
            if (p->affine)
                score_affine(p, &P, qp, tp);
            else
                score_linear(p, &P, qp, tp);
            pair_max[(size_t)qi * nt + ti] = P.max;
            int before = sink.n;
            if (sink.n + (int)cells > sink.cap) {
                while (sink.n + (int64_t)cells > sink.cap) sink.cap *= 2;
                sink.starts = (orc_start*)realloc(sink.starts, sizeof(orc_start) * sink.cap);
                sink.keys = (start_key*)realloc(sink.keys, sizeof(start_key) * sink.cap);
            }
            traceback_pair(p, &P, pos_score[(size_t)ti * nq + qi], (uint32_t)qi, (uint32_t)ti, &sink);
            (void)before;
            zc[(size_t)qi * nt + ti] = P.zc;
            zX[(size_t)qi * nt + ti] = P.X;
            zY[(size_t)qi * nt + ti] = P.Y;
            free(P.H);
            free(P.I);
            free(P.J);
            free(P.dir);
            free(qp);
            free(tp);
        }
    }

    /* starts in emission order, then the host walk's stable ascending sort
     * by score (SmithWaterman.py:699) */
    *n_starts = sink.n;
    for (int64_t s = 0; s < sink.n && s < max_starts; ++s) starts_out[s] = sink.starts[s];
    if (sink.n > max_starts) rc = -1;
    /* the host reads the first start_cap starting points of the device
     * buffer (emission order) when there are at least that many
     * (SmithWaterman.py:683-687), then sorts those by score (:699) */
    int64_t walk_n = sink.n;
    if (start_cap >= 0 && walk_n >= start_cap) {
        qsort(sink.keys, sink.n, sizeof(start_key), emit_cmp);
        walk_n = start_cap;
    }
    qsort(sink.keys, walk_n, sizeof(start_key), key_cmp);

    int64_t nh = 0, used = 0;
    for (int64_t s = 0; s < walk_n; ++s) {
        const orc_start* st = &sink.starts[sink.keys[s].src];
        int qi = (int)st->sequence, ti = (int)st->target;
        uint8_t* Z = zc[(size_t)qi * nt + ti];
        int Y = zY[(size_t)qi * nt + ti];
        const uint8_t* qs = q_res + q_off[qi];
        const uint8_t* ts = t_res + t_off[ti];
        int bx = (int)st->block_x, by = (int)st->block_y, vx = (int)st->value_x, vy = (int)st->value_y;
        int s_end = bx * SHARED + vx, t_end = by * SHARED + vy;
        int s_start = s_end + 1, t_start = t_end + 1;
        int matches = 0, mismatches = 0, ncols = 0;
        int lq = (int)(q_off[qi + 1] - q_off[qi]), lt = (int)(t_off[ti + 1] - t_off[ti]);
        char* sq = (char*)malloc(lq + lt + 2);
        char* al = (char*)malloc(lq + lt + 2);
        char* tg = (char*)malloc(lq + lt + 2);
#define ZC(X_, Y_) Z[(size_t)(X_) * Y + (Y_)]
        int direction = ZC(bx * SHARED + vx, by * SHARED + vy);
        int show = 1;
        if (q_idkey[qi] == t_idkey[ti]) { /* :752-755 */
            direction = STOP_DIRECTION;
            show = 0;
        }
        if ((double)st->score < host_min_score) show = 0; /* :758-759 */
        while (show && bx >= 0 && by >= 0 && vx >= 0 && vy >= 0 && direction != STOP_DIRECTION &&
               direction != NO_DIRECTION) { /* :761-821 */
            int cx = bx * SHARED + vx, cy = by * SHARED + vy;
            direction = ZC(cx, cy);
            ZC(cx, cy) = IN_ALIGNMENT;
            if (direction == IN_ALIGNMENT) {
                show = 0;
            } else if (direction == UPPER_LEFT || direction == STOP_DIRECTION) {
                char a = (char)ts[cy], b = (char)qs[cx];
                tg[ncols] = a;
                sq[ncols] = b;
                int eq = (a | 0x20) == (b | 0x20) && ((a >= 'A' && a <= 'Z') || (a >= 'a' && a <= 'z'))
                             ? 1
                             : a == b;
                al[ncols] = eq ? '|' : '.';
                s_start--;
                t_start--;
                if (eq) matches++; else mismatches++;
                if (direction == UPPER_LEFT) {
                    if (vx == 0) { bx--; vx = SHARED - 1; } else vx--;
                    if (vy == 0) { by--; vy = SHARED - 1; } else vy--;
                }
                ncols++;
            } else if (direction == LEFT) {
                tg[ncols] = '-';
                sq[ncols] = (char)qs[cx];
                al[ncols] = ' ';
                s_start--;
                if (vx == 0) { bx--; vx = SHARED - 1; } else vx--;
                ncols++;
            } else if (direction == UPPER) {
                tg[ncols] = (char)ts[cy];
                sq[ncols] = '-';
                al[ncols] = ' ';
                t_start--;
                if (vy == 0) { by--; vy = SHARED - 1; } else vy--;
                ncols++;
            } else {
                bx = -1;
            }
        }
#undef ZC
        (void)lt;
        if (show) {
            if (nh < max_hits && used + 3 * (int64_t)ncols <= strbuf_cap) {
                orc_hit* h = &hits[nh];
                h->query = qi;
                h->target = ti;
                h->s_start = s_start;
                h->s_end = s_end;
                h->t_start = t_start;
                h->t_end = t_end;
                h->score = st->score;
                h->matches = matches;
                h->mismatches = mismatches;
                h->n_cols = ncols;
                h->str_offset = used;
                /* strings were built backwards; the reference reverses them (:827-832) */
                for (int c = 0; c < ncols; ++c) {
                    strbuf[used + c] = sq[ncols - 1 - c];
                    strbuf[used + ncols + c] = al[ncols - 1 - c];
                    strbuf[used + 2 * ncols + c] = tg[ncols - 1 - c];
                }
            } else {
                rc = -1;
            }
            nh++;
            used += 3 * (int64_t)ncols;
        }
        free(sq);
        free(al);
        free(tg);
    }
    *n_hits = nh;
    *str_used = used;
    for (size_t k = 0; k < (size_t)nq * nt; ++k) free(zc[k]);
    free(zc);
    free(zX);
    free(zY);
    free(sink.starts);
    free(sink.keys);
    return rc;
}

/* Score-only restatement: the pair maxima of calculateScore[AffineGap]. */
void orc_pair_max(const orc_params* p, int nq, const uint8_t* q_res, const int64_t* q_off, int nt,
                  const uint8_t* t_res, const int64_t* t_off, float* pair_max) {
    for (int ti = 0; ti < nt; ++ti) {
        for (int qi = 0; qi < nq; ++qi) {
            int lq = (int)(q_off[qi + 1] - q_off[qi]), lt = (int)(t_off[ti + 1] - t_off[ti]);
            pair_mats P;
            P.X = (lq + SHARED - 1) / SHARED * SHARED;
            P.Y = (lt + SHARED - 1) / SHARED * SHARED;
            if (P.X == 0) P.X = SHARED;
            if (P.Y == 0) P.Y = SHARED;
            size_t cells = (size_t)P.X * P.Y;
            uint8_t* qp = (uint8_t*)calloc(P.X, 1);
            uint8_t* tp = (uint8_t*)calloc(P.Y, 1);
            memcpy(qp, q_res + q_off[qi], lq);
            memcpy(tp, t_res + t_off[ti], lt);
            P.H = (float*)calloc(cells, 4);
            P.I = p->affine ? (float*)calloc(cells, 4) : NULL;
            P.J = p->affine ? (float*)calloc(cells, 4) : NULL;
            P.dir = (uint8_t*)calloc(cells, 1);
            P.zc = NULL;
            if (p->affine)
                score_affine(p, &P, qp, tp);
            else
                score_linear(p, &P, qp, tp);
            pair_max[(size_t)qi * nt + ti] = P.max;
            free(P.H);
            free(P.I);
            free(P.J);
            free(P.dir);
            free(qp);
            free(tp);
        }
    }
}
