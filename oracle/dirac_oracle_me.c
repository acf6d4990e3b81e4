/*
 * dirac_oracle_me.c -- TEST INFRASTRUCTURE ONLY (see dirac_oracle.h).
 *
 * Plain-C restatement of the reference's motion estimation for one picture: the pel-accurate
 * hierarchical block matching (PixelMatcher, libdirac_motionest/pixel_match.cpp), the
 * Lagrangian lambda map (MEData::SetLambdaMap, libdirac_common/motion.cpp:128-196), sub-pel
 * refinement (SubpelRefine / BlockMatcher::RefineMatchSubp, me_subpel.cpp, block_match.cpp)
 * and superblock mode decision with DC estimation (ModeDecider, me_mode_decn.cpp).
 *
 * Floating-point decisions follow the reference's operation order in float (costs), double
 * (the 1.1 / 0.85 / 4.0 factors) and long double (transition statistics), so the decisions
 * match bit for bit on the same host.  Candidate search keeps the reference's candidate
 * order; the first strictly smaller cost wins, as there.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dirac_oracle.h"

typedef struct {
    int x, y;
} mvec;

typedef struct {
    float SAD, mvcost, total;
} mvcost_t;

typedef struct {
    int xblen, yblen, xbsep, ybsep, xoff, yoff;
} olb_t;

/* One MEData: per-unit vectors and costs for up to two references, modes, DC, lambdas. */
typedef struct {
    int xnb, ynb;
    mvec* mv[2];
    mvcost_t* cost[2];
    mvcost_t* bicost;
    float* intra;
    uint8_t* mode;
    int16_t* dc[3];
    float* lambda;
} medata;

static int imin(int a, int b) { return a < b ? a : b; }
static int imax(int a, int b) { return a > b ? a : b; }
static int bchk(int v, int n) { return v < 0 ? 0 : (v >= n ? n - 1 : v); }
static int norm1(mvec a) { return abs(a.x) + abs(a.y); }
static mvec mvsub(mvec a, mvec b) { mvec r = {a.x - b.x, a.y - b.y}; return r; }
static mvec mvshl(mvec a, int s) { mvec r = {a.x << s, a.y << s}; return r; }

static olb_t make_olb(int xblen, int yblen, int xbsep, int ybsep) {
    olb_t o = {xblen, yblen, xbsep, ybsep, (xblen - xbsep) / 2, (yblen - ybsep) / 2};
    return o;
}

/* PicturePredParams::SetBlockSizes (common.cpp:305-315): levels 1 and 0 (sub-superblocks,
 * superblocks); note that their heights grow by the horizontal separation. */
static void luma_levels(const orc_block_params* bp, olb_t lb[3]) {
    lb[2] = make_olb(bp->xblen, bp->yblen, bp->xbsep, bp->ybsep);
    lb[1] = make_olb(lb[2].xblen + lb[2].xbsep, lb[2].yblen + lb[2].xbsep, 2 * lb[2].xbsep, 2 * lb[2].ybsep);
    lb[0] = make_olb(lb[1].xblen + lb[1].xbsep, lb[1].yblen + lb[1].xbsep, 2 * lb[1].xbsep, 2 * lb[1].ybsep);
}

static int medata_init(medata* m, int xnb, int ynb) {
    memset(m, 0, sizeof(*m));
    m->xnb = xnb;
    m->ynb = ynb;
    const size_t n = (size_t)xnb * ynb;
    for (int r = 0; r < 2; ++r) {
        m->mv[r] = (mvec*)calloc(n, sizeof(mvec));
        m->cost[r] = (mvcost_t*)calloc(n, sizeof(mvcost_t));
        if (!m->mv[r] || !m->cost[r]) return -5;
    }
    m->bicost = (mvcost_t*)calloc(n, sizeof(mvcost_t));
    m->intra = (float*)calloc(n, sizeof(float));
    m->mode = (uint8_t*)calloc(n, 1);
    m->lambda = (float*)calloc(n, sizeof(float));
    for (int c = 0; c < 3; ++c) m->dc[c] = (int16_t*)calloc(n, sizeof(int16_t));
    if (!m->bicost || !m->intra || !m->mode || !m->lambda || !m->dc[0] || !m->dc[1] || !m->dc[2]) return -5;
    return 0;
}

static void medata_free(medata* m) {
    for (int r = 0; r < 2; ++r) {
        free(m->mv[r]);
        free(m->cost[r]);
    }
    free(m->bicost);
    free(m->intra);
    free(m->mode);
    free(m->lambda);
    for (int c = 0; c < 3; ++c) free(m->dc[c]);
}

/* BlockDiffParams::SetBlockLimits (me_utils.cpp:58-80); lengths may come out <= 0. */
typedef struct {
    int xp, yp, xl, yl;
} blim;

static blim block_limits(const olb_t* o, int pw, int ph, int bx, int by) {
    blim b;
    const int lx = bx * o->xbsep - o->xoff, ly = by * o->ybsep - o->yoff;
    b.xp = imax(lx, 0);
    b.yp = imax(ly, 0);
    b.xl = o->xblen - b.xp + lx;
    b.yl = o->yblen - b.yp + ly;
    if (b.xp + b.xl - 1 > pw - 1) b.xl = pw - b.xp;
    if (b.yp + b.yl - 1 > ph - 1) b.yl = ph - b.yp;
    return b;
}

/* MvMedian of three vectors / MvMean of two (motion.cpp:502-521, 667-681). */
static int med3(int a, int b, int c) { return a + b + c - imax(imax(a, b), c) - imin(imin(a, b), c); }
static mvec mv_median3(mvec a, mvec b, mvec c) {
    mvec r = {med3(a.x, b.x, c.x), med3(a.y, b.y, c.y)};
    return r;
}
static mvec mv_mean(mvec a, mvec b) {
    mvec r = {(a.x + b.x + 1) >> 1, (a.y + b.y + 1) >> 1};
    return r;
}
/* MvMedian of 0-4 vectors (motion.cpp:560-600). */
static mvec mv_median_list(const mvec* v, int n) {
    mvec r = {0, 0};
    if (n == 1) return v[0];
    if (n == 2) return mv_mean(v[0], v[1]);
    if (n == 3) return mv_median3(v[0], v[1], v[2]);
    if (n == 4) {
        int sx = 0, sy = 0, mxx = v[0].x, mnx = v[0].x, mxy = v[0].y, mny = v[0].y;
        for (int i = 0; i < 4; ++i) {
            sx += v[i].x;
            sy += v[i].y;
            mxx = imax(mxx, v[i].x);
            mnx = imin(mnx, v[i].x);
            mxy = imax(mxy, v[i].y);
            mny = imin(mny, v[i].y);
        }
        r.x = (sx - (mxx + mnx) + 1) >> 1;
        r.y = (sy - (mxy + mny) + 1) >> 1;
    }
    return r;
}

/* ---------------------------------------------------------------------------------------- */
/* Candidate lists (block_match.cpp:48-190)                                                  */
/* ---------------------------------------------------------------------------------------- */

#define MAX_CANDS 1200

typedef struct {
    mvec c[MAX_CANDS];
    int n;         /* candidates in all lists */
    int zero_len;  /* length of the persistent zero-centred list */
} cand_list;

static void add_vect(cand_list* L, mvec v) {
    for (int i = 0; i < L->n; ++i)
        if (L->c[i].x == v.x && L->c[i].y == v.y) return;
    if (L->n < MAX_CANDS) L->c[L->n++] = v;
}

/* AddNewVlist: centre, then (+-i, 0) for i = 1..xr, then rows +-j with i = -xr..xr;
 * duplicates of any earlier candidate are dropped. */
static void add_new_vlist(cand_list* L, mvec mv, int xr, int yr) {
    mvec t = mv;
    add_vect(L, t);
    for (int i = 1; i <= xr; ++i) {
        t.x = mv.x + i;
        add_vect(L, t);
        t.x = mv.x - i;
        add_vect(L, t);
    }
    for (int j = 1; j <= yr; ++j)
        for (int i = -xr; i <= xr; ++i) {
            t.x = mv.x + i;
            t.y = mv.y + j;
            add_vect(L, t);
            t.y = mv.y - j;
            add_vect(L, t);
        }
}

/* ---------------------------------------------------------------------------------------- */
/* Block differences (me_utils.cpp)                                                         */
/* ---------------------------------------------------------------------------------------- */

/* PelBlockDiff: SAD against a same-size reference, reference coordinates clamped. */
static int pel_sad(const int16_t* pic, const int16_t* ref, int pw, int ph, blim b, mvec mv) {
    int sum = 0;
    for (int j = b.yp; j < b.yp + b.yl; ++j) {
        const int16_t* pr = pic + (size_t)j * pw;
        const int16_t* rr = ref + (size_t)bchk(j + mv.y, ph) * pw;
        for (int i = b.xp; i < b.xp + b.xl; ++i) sum += abs((int16_t)(pr[i] - rr[bchk(i + mv.x, pw)]));
    }
    return sum;
}

/* Prediction sample from an upconverted reference (uw x uh) at precision level p
 * (1 half, 2 quarter, 3 eighth), coordinates clamped to the upconverted array. */
static int up_pred(const int16_t* up, int uw, int uh, int p, int x, int y, mvec mv) {
#define U(yy, xx) ((int)up[(size_t)bchk((yy), uh) * uw + bchk((xx), uw)])
    if (p == 1) return U(2 * y + mv.y, 2 * x + mv.x);
    if (p == 2) {
        const int rx = mv.x & 1, ry = mv.y & 1;
        const int bx = 2 * x + (mv.x >> 1), by = 2 * y + (mv.y >> 1);
        return ((2 - rx) * (2 - ry) * U(by, bx) + rx * (2 - ry) * U(by, bx + 1) + (2 - rx) * ry * U(by + 1, bx) +
                rx * ry * U(by + 1, bx + 1) + 2) >> 2;
    }
    {
        const int rx = mv.x & 3, ry = mv.y & 3;
        const int bx = 2 * x + (mv.x >> 2), by = 2 * y + (mv.y >> 2);
        return ((4 - rx) * (4 - ry) * U(by, bx) + rx * (4 - ry) * U(by, bx + 1) + (4 - rx) * ry * U(by + 1, bx) +
                rx * ry * U(by + 1, bx + 1) + 8) >> 4;
    }
#undef U
}

/* BlockDiff{Half,Quarter,Eighth}Pel::Diff without cost: float sum of |pred - pic| in raster order. */
static float subpel_sum(const int16_t* pic, int pw, const int16_t* up, int uw, int uh, int p, blim b, mvec mv) {
    if (b.xl <= 0 || b.yl <= 0) return 0.0f;
    float sum = 0.0f;
    for (int y = b.yp; y < b.yp + b.yl; ++y)
        for (int x = b.xp; x < b.xp + b.xl; ++x)
            sum += (float)abs(up_pred(up, uw, uh, p, x, y, mv) - pic[(size_t)y * pw + x]);
    return sum;
}

/* The same with cost: sum starts at mvcost*lambda; the candidate replaces the best when its
 * total is strictly smaller (the reference's per-row early exit is equivalent, as float sums
 * of non-negative terms never decrease). */
static void subpel_try(const int16_t* pic, int pw, const int16_t* up, int uw, int uh, int p, blim b, mvec mv,
                       float mvcost, float lambda, mvcost_t* best, mvec* best_mv) {
    if (b.xl <= 0 || b.yl <= 0) return;
    const float start = mvcost * lambda;
    float sum = start;
    for (int y = b.yp; y < b.yp + b.yl; ++y)
        for (int x = b.xp; x < b.xp + b.xl; ++x)
            sum += (float)abs(up_pred(up, uw, uh, p, x, y, mv) - pic[(size_t)y * pw + x]);
    if (sum < best->total) {
        *best_mv = mv;
        best->total = sum;
        best->mvcost = mvcost;
        best->SAD = sum - start;
    }
}

/* BiBlock*Pel::Diff: |((2 pic - p1) - p2) >> 1| with int16 intermediates, summed in float.
 * Eighth-pel quirk reproduced: when the second reference's block needs bounds checking,
 * BiBlockEighthPel::Diff walks it from the FIRST reference's integer start position (with
 * the second vector's fractional weights), me_utils.cpp:1764-1768. */
static float bi_sum(const int16_t* pic, int pw, const int16_t* up1, const int16_t* up2, int uw, int uh, int p,
                    blim b, mvec mv1, mvec mv2) {
    if (b.xl <= 0 || b.yl <= 0) return 0.0f;
    mvec m2 = mv2;
    if (p == 3) {
        const int sx = (b.xp << 1) + (mv2.x >> 2), sy = (b.yp << 1) + (mv2.y >> 2);
        if (sx < 0 || sx + (b.xl << 1) >= uw || sy < 0 || sy + (b.yl << 1) >= uh) {
            /* same fractional part as mv2, integer part of mv1 */
            m2.x = ((mv1.x >> 2) << 2) | (mv2.x & 3);
            m2.y = ((mv1.y >> 2) << 2) | (mv2.y & 3);
        }
    }
    float sum = 0.0f;
    for (int y = b.yp; y < b.yp + b.yl; ++y)
        for (int x = b.xp; x < b.xp + b.xl; ++x) {
            const int16_t d = (int16_t)((pic[(size_t)y * pw + x] << 1) - up_pred(up1, uw, uh, p, x, y, mv1));
            const int16_t t = (int16_t)((d - up_pred(up2, uw, uh, p, x, y, m2)) >> 1);
            sum += (float)abs(t);
        }
    return sum;
}

/* IntraBlockDiff::CalcDC / Diff: truncating mean, then SAD against it. */
static int16_t block_dc(const int16_t* pic, int pw, blim b) {
    if (b.xl <= 0 || b.yl <= 0) return 0;
    int s = 0;
    for (int y = b.yp; y < b.yp + b.yl; ++y)
        for (int x = b.xp; x < b.xp + b.xl; ++x) s += pic[(size_t)y * pw + x];
    s /= b.xl * b.yl;
    return (int16_t)s;
}

static float intra_diff(const int16_t* pic, int pw, blim b, int16_t* dc) {
    if (b.xl <= 0 || b.yl <= 0) {
        *dc = 0;
        return 0.0f;
    }
    *dc = block_dc(pic, pw, b);
    int s = 0;
    for (int y = b.yp; y < b.yp + b.yl; ++y)
        for (int x = b.xp; x < b.xp + b.xl; ++x) s += abs(pic[(size_t)y * pw + x] - *dc);
    return (float)s;
}

/* ---------------------------------------------------------------------------------------- */
/* Pel-accurate hierarchical search (pixel_match.cpp:59-380)                                  */
/* ---------------------------------------------------------------------------------------- */

static void find_best_pel(const int16_t* pic, const int16_t* ref, int pw, int ph, const olb_t* o, medata* md,
                          int r, int bx, int by, const cand_list* L, mvec pred) {
    const size_t k = (size_t)by * md->xnb + bx;
    const blim b = block_limits(o, pw, ph, bx, by);
    float best_cost = md->cost[r][k].total;
    mvec best_mv = md->mv[r][k];
    if (b.xl > 0 && b.yl > 0) {
        for (int i = 0; i < L->n; ++i) {
            const int sad = pel_sad(pic, ref, pw, ph, b, L->c[i]);
            if ((float)sad < best_cost) {
                best_cost = (float)sad;
                best_mv = L->c[i];
            }
        }
    }
    md->mv[r][k] = best_mv;
    md->cost[r][k].SAD = best_cost;
    md->cost[r][k].mvcost = (float)norm1(mvsub(best_mv, pred));
    md->cost[r][k].total = md->cost[r][k].SAD + 0.0f * md->cost[r][k].mvcost;
}

static void match_pic_pel(const int16_t* pic, const int16_t* ref, int pw, int ph, const olb_t* o, medata* md,
                          const medata* guide, int r, int level, int depth, cand_list* L) {
    const int rad = imin(level + 1, 5);
    const int n = md->xnb * md->ynb;
    for (int i = 0; i < n; ++i) {
        md->mv[r][i].x = md->mv[r][i].y = 0;
        md->cost[r][i].total = 10000000.0f;
    }
    L->n = 0;
    const mvec zero = {0, 0};
    add_new_vlist(L, zero, rad, rad);
    L->zero_len = L->n;
    for (int by = 0; by < md->ynb; ++by) {
        for (int bx = 0; bx < md->xnb; ++bx) {
            mvec pred = {0, 0};
            const mvec* mv = md->mv[r];
            const int W = md->xnb;
            if (by == 0) {
                if (bx > 0) pred = mv[bx - 1];
            } else if (bx == 0) {
                pred = mv[(size_t)(by - 1) * W];
            } else if (bx < W - 1) {
                pred = mv_median3(mv[(size_t)by * W + bx - 1], mv[(size_t)(by - 1) * W + bx],
                                  mv[(size_t)(by - 1) * W + bx + 1]);
            } else {
                pred = mv_mean(mv[(size_t)(by - 1) * W + bx], mv[(size_t)by * W + bx - 1]);
            }
            if (level < depth) {
                const int gx = bchk(bx >> 1, guide->xnb), gy = bchk(by >> 1, guide->ynb);
                const mvec g = guide->mv[r][(size_t)gy * guide->xnb + gx];
                const mvec g2 = {g.x * 2, g.y * 2};
                add_new_vlist(L, g2, rad, rad);
            }
            add_new_vlist(L, pred, rad, rad);
            find_best_pel(pic, ref, pw, ph, o, md, r, bx, by, L, pred);
            L->n = L->zero_len;
        }
    }
}

/* ---------------------------------------------------------------------------------------- */
/* Lambda map (motion.cpp:128-196, 201-333)                                                   */
/* ---------------------------------------------------------------------------------------- */

/* FindTransitions: the vector-variation map (the SAD-based map computed first is overwritten
 * in the reference, so it has no effect), widened to whole superblocks. */
static void find_transitions(const medata* md, int r, uint8_t* trans) {
    const int W = md->xnb, H = md->ynb;
    double* val = (double*)calloc((size_t)W * H, sizeof(double));
    long double total = 0.0;
    for (int j = 1; j < H - 1; ++j)
        for (int i = 1; i < W - 1; ++i) {
            double v = 0.0;
            const mvec c = md->mv[r][(size_t)j * W + i];
            for (int q = -1; q <= 1; ++q)
                for (int p = -1; p <= 1; ++p) {
                    const double d = (double)norm1(mvsub(md->mv[r][(size_t)(j + q) * W + i + p], c));
                    if (d > v) v = d;
                }
            val[(size_t)j * W + i] = v;
            total += v;
        }
    const long double mean = total / (long double)(W * H);
    long double sd = 0.0;
    for (int j = 1; j < H - 1; ++j)
        for (int i = 1; i < W - 1; ++i) {
            double diff = (double)(val[(size_t)j * W + i] - mean);
            diff *= diff;
            sd += diff;
        }
    sd /= (long double)(W * H);
    sd = sqrtl(sd);
    const double threshold = (double)(mean + 3 * sd);
    for (int k = 0; k < W * H; ++k) trans[k] = val[k] >= threshold;
    for (int j = 0; j < H / 4; ++j)
        for (int i = 0; i < W / 4; ++i) {
            int any = 0;
            for (int q = 4 * j; q < 4 * (j + 1); ++q)
                for (int p = 4 * i; p < 4 * (i + 1); ++p) any |= trans[(size_t)q * W + p];
            for (int q = 4 * j; q < 4 * (j + 1); ++q)
                for (int p = 4 * i; p < 4 * (i + 1); ++p) trans[(size_t)q * W + p] = (uint8_t)any;
        }
    free(val);
}

static void set_lambda_map(medata* md, int nref, float lambda) {
    const int W = md->xnb, H = md->ynb;
    uint8_t* t1 = (uint8_t*)calloc((size_t)W * H, 1);
    uint8_t* t2 = (uint8_t*)calloc((size_t)W * H, 1);
    find_transitions(md, 0, t1);
    if (nref > 1) find_transitions(md, 1, t2);
    for (int j = 0; j < H; ++j)
        for (int i = 0; i < W; ++i) {
            const size_t k = (size_t)j * W + i;
            float l;
            if (nref == 1) {
                l = t1[k] ? 0.0f : lambda;
            } else {
                if (t1[k] && t2[k])
                    l = 0.0f;
                else if (t1[k] || t2[k])
                    l = (float)(lambda / 4.0);
                else
                    l = lambda;
            }
            if (i < 4 || j < 4) l = (float)(l / 5.0);
            md->lambda[k] = l;
        }
    free(t1);
    free(t2);
}

/* SetLambdaMap(level, block map, wt): max over the covered blocks, times wt. */
static void set_lambda_map_level(medata* md, int level, const medata* blocks, float wt) {
    const int f = 1 << (2 - level);
    for (int j = 0; j < md->ynb; ++j)
        for (int i = 0; i < md->xnb; ++i) {
            float l = blocks->lambda[(size_t)(f * j) * blocks->xnb + f * i];
            for (int q = f * j; q < f * (j + 1); ++q)
                for (int p = f * i; p < f * (i + 1); ++p) {
                    const float v = blocks->lambda[(size_t)q * blocks->xnb + p];
                    if (v > l) l = v;
                }
            md->lambda[(size_t)j * md->xnb + i] = l * wt;
        }
}

/* ---------------------------------------------------------------------------------------- */
/* Sub-pel refinement (me_subpel.cpp:65-176, block_match.cpp:327-467)                         */
/* ---------------------------------------------------------------------------------------- */

static int getvarup(mvec pred, mvec mv) { return imin(norm1(mvsub(mv, pred)), norm1(mv)); }

static void refine_block(const int16_t* pic, int pw, int ph, const int16_t* up, const olb_t* o, medata* md, int r,
                         int bx, int by, mvec pred, float lambda, int prec) {
    const size_t k = (size_t)by * md->xnb + bx;
    const int uw = 2 * pw, uh = 2 * ph;
    const blim b = block_limits(o, pw, ph, bx, by);
    mvcost_t* cost = &md->cost[r][k];
    cost->mvcost = (float)getvarup(pred, mvshl(md->mv[r][k], prec));
    cost->total = cost->SAD + lambda * cost->mvcost;
    mvcost_t best = *cost;
    mvec best_mv = md->mv[r][k];
    if (best.SAD < (float)(2 * b.xl * b.yl)) {
        md->mv[r][k] = mvshl(md->mv[r][k], prec);
        return;
    }
    mvcost_t pc;
    pc.mvcost = 0.0f;
    pc.SAD = subpel_sum(pic, pw, up, uw, uh, prec, b, pred);
    pc.total = pc.SAD;
    if (pc.SAD < (float)(2 * b.xl * b.yl)) {
        md->mv[r][k] = pred;
        *cost = pc;
        return;
    }
    for (int i = 1; i <= prec; ++i) {
        best_mv = mvshl(best_mv, 1);
        mvec tb = best_mv;
        const mvec nb[4] = {{best_mv.x - 1, best_mv.y}, {best_mv.x + 1, best_mv.y},
                            {best_mv.x, best_mv.y - 1}, {best_mv.x, best_mv.y + 1}};
        for (int q = 0; q < 4; ++q)
            subpel_try(pic, pw, up, uw, uh, i, b, nb[q], (float)getvarup(pred, mvshl(nb[q], prec - i)), lambda, &best,
                       &tb);
        if (tb.x != best_mv.x) {
            const mvec nbest = tb;
            const mvec c2[2] = {{nbest.x, nbest.y - 1}, {nbest.x, nbest.y + 1}};
            for (int q = 0; q < 2; ++q)
                subpel_try(pic, pw, up, uw, uh, i, b, c2[q], (float)getvarup(pred, mvshl(c2[q], prec - i)), lambda,
                           &best, &tb);
        } else if (tb.y != best_mv.y) {
            const mvec nbest = tb;
            const mvec c2[2] = {{nbest.x - 1, nbest.y}, {nbest.x + 1, nbest.y}};
            for (int q = 0; q < 2; ++q)
                subpel_try(pic, pw, up, uw, uh, i, b, c2[q], (float)getvarup(pred, mvshl(c2[q], prec - i)), lambda,
                           &best, &tb);
        }
        best_mv = tb;
        if ((double)best.total > 1.1 * (double)pc.total) {
            md->mv[r][k] = pred;
            *cost = pc;
            return;
        }
    }
    md->mv[r][k] = best_mv;
    *cost = best;
}

static void subpel_pic(const int16_t* pic, int pw, int ph, const int16_t* up, const olb_t* o, medata* md, int r,
                       int prec) {
    static const int nsx[4] = {-1, -1, 0, 1}, nsy[4] = {0, -1, -1, -1};
    const int W = md->xnb, H = md->ynb;
    for (int by = 0; by < H; ++by)
        for (int bx = 0; bx < W; ++bx) {
            mvec nbr[4];
            int n = 0;
            for (int i = 0; i < 4; ++i) {
                const int x = bx + nsx[i], y = by + nsy[i];
                const int all = bx > 0 && by > 0 && bx < W - 1;
                if (all || (x >= 0 && y >= 0 && x < W && y < H)) nbr[n++] = md->mv[r][(size_t)y * W + x];
            }
            const mvec pred = mv_median_list(nbr, n);
            refine_block(pic, pw, ph, up, o, md, r, bx, by, pred, md->lambda[(size_t)by * W + bx], prec);
        }
}

/* ---------------------------------------------------------------------------------------- */
/* Mode decision (me_mode_decn.cpp:66-573)                                                    */
/* ---------------------------------------------------------------------------------------- */

typedef struct {
    const int16_t* pic;
    int pw, ph;
    const int16_t* up[2];
    int nref, prec;
    olb_t lb[3];
    float level_factor[3];
    medata* set[3];
    float* sbcost;
    uint8_t* split;
    int xnsb, ynsb;
} mode_ctx;

static void find_best_subp(const mode_ctx* M, int level, int r, int x, int y, const mvec* cands, int nc, mvec pred,
                           float lambda) {
    medata* md = M->set[level];
    const size_t k = (size_t)y * md->xnb + x;
    const blim b = block_limits(&M->lb[level], M->pw, M->ph, x, y);
    mvcost_t best = md->cost[r][k];
    best.total = 100000000.0f;
    mvec best_mv = md->mv[r][k];
    for (int i = 0; i < nc; ++i)
        subpel_try(M->pic, M->pw, M->up[r], 2 * M->pw, 2 * M->ph, M->prec, b, cands[i],
                   (float)getvarup(pred, cands[i]), lambda, &best, &best_mv);
    md->mv[r][k] = best_mv;
    md->cost[r][k] = best;
}

static void do_me(mode_ctx* M, int x, int y, int level) {
    medata* md = M->set[level];
    const medata* guide = M->set[level + 1];
    const medata* blk = M->set[2];
    const int gx = x << 1, gy = y << 1;
    const int xb = x << (2 - level), yb = y << (2 - level);
    const float lambda = md->lambda[(size_t)y * md->xnb + x];
    for (int r = 0; r < M->nref; ++r) {
        /* four single-vector lists from the guide level, duplicates dropped */
        mvec c[4];
        int nc = 0;
        for (int j = 0; j < 2; ++j)
            for (int i = 0; i < 2; ++i) {
                const mvec v = guide->mv[r][(size_t)(gy + j) * guide->xnb + gx + i];
                int dup = 0;
                for (int q = 0; q < nc; ++q) dup |= (c[q].x == v.x && c[q].y == v.y);
                if (!dup) c[nc++] = v;
            }
        const mvec* bv = blk->mv[r];
        const int W = blk->xnb;
        mvec pred = {0, 0};
        if (xb > 0 && yb > 0)
            pred = mv_median3(bv[(size_t)yb * W + xb - 1], bv[(size_t)(yb - 1) * W + xb - 1], bv[(size_t)(yb - 1) * W + xb]);
        else if (xb == 0 && yb > 0)
            pred = mv_mean(bv[(size_t)(yb - 1) * W + xb], bv[(size_t)(yb - 1) * W + xb + 1]);
        else if (xb > 0 && yb == 0)
            pred = mv_mean(bv[(size_t)yb * W + xb - 1], bv[(size_t)(yb + 1) * W + xb - 1]);
        md->cost[r][(size_t)y * md->xnb + x].total = 100000000.0f;
        find_best_subp(M, level, r, x, y, c, nc, pred, lambda);
    }
}

static float do_unit_decn(mode_ctx* M, int x, int y, int level) {
    medata* md = M->set[level];
    const size_t k = (size_t)y * md->xnb + x;
    const float lambda = md->lambda[k];
    const float mode_cost = 0.0f;
    const blim b = block_limits(&M->lb[level], M->pw, M->ph, x, y);
    md->mode[k] = 1; /* REF1_ONLY */
    md->cost[0][k].total *= M->level_factor[level];
    float min_cost = md->cost[0][k].total + mode_cost;
    float best_sad = md->cost[0][k].SAD;
    if (M->nref > 1) {
        md->cost[1][k].total *= M->level_factor[level];
        float unit = md->cost[1][k].total + mode_cost;
        if (unit < min_cost) {
            md->mode[k] = 2;
            min_cost = unit;
            best_sad = md->cost[1][k].SAD;
        }
        mvcost_t* bc = &md->bicost[k];
        bc->mvcost = md->cost[0][k].mvcost + md->cost[1][k].mvcost;
        bc->SAD = bi_sum(M->pic, M->pw, M->up[0], M->up[1], 2 * M->pw, 2 * M->ph, M->prec, b, md->mv[0][k],
                         md->mv[1][k]);
        bc->total = bc->SAD + lambda * bc->mvcost;
        bc->total *= M->level_factor[level];
        unit = bc->total + mode_cost;
        if (unit < min_cost) {
            md->mode[k] = 3;
            min_cost = unit;
            best_sad = bc->SAD;
        }
    }
    if (level == 2 && (double)best_sad > 4.0 * M->lb[level].xblen * M->lb[level].yblen) {
        md->intra[k] = intra_diff(M->pic, M->pw, b, &md->dc[0][k]);
        md->intra[k] *= M->level_factor[level];
        const float unit = md->intra[k] + mode_cost;
        if (unit < min_cost && (double)md->intra[k] < 0.85 * (double)best_sad) {
            md->mode[k] = 0;
            min_cost = unit;
        }
    }
    return min_cost;
}

static void do_level_decn(mode_ctx* M, int xsb, int ysb, int level) {
    const int xs = xsb << level, ys = ysb << level;
    const int xe = xs + (1 << level), ye = ys + (1 << level);
    const size_t sb = (size_t)ysb * M->xnsb + xsb;
    float sb_cost = 0.0f;
    for (int j = ys; j < ye; ++j)
        for (int i = xs; i < xe; ++i) {
            if (level < 2) do_me(M, i, j, level);
            sb_cost += do_unit_decn(M, i, j, level);
        }
    if (level == 2) {
        M->split[sb] = 2;
        M->sbcost[sb] = sb_cost;
    }
    if (level < 2 && sb_cost <= M->sbcost[sb]) {
        M->sbcost[sb] = sb_cost;
        M->split[sb] = (uint8_t)level;
        medata* lv = M->set[level];
        medata* bl = M->set[2];
        for (int j = ys; j < ye; ++j)
            for (int i = xs; i < xe; ++i) {
                const size_t src = (size_t)j * lv->xnb + i;
                for (int v = j << (2 - level); v < (j + 1) << (2 - level); ++v)
                    for (int u = i << (2 - level); u < (i + 1) << (2 - level); ++u) {
                        const size_t dst = (size_t)v * bl->xnb + u;
                        bl->mode[dst] = lv->mode[src];
                        bl->dc[0][dst] = lv->dc[0][src];
                        bl->mv[0][dst] = lv->mv[0][src];
                        if (M->nref > 1) bl->mv[1][dst] = lv->mv[1][src];
                    }
            }
    }
}

/* ModeDecider::SetDC (me_mode_decn.cpp:540-573): block DCs, 3x3-smoothed except on the first
 * row / column and the last column; the last row keeps its previous contents. */
static void set_dc(const int16_t* pic, int pw, int ph, const olb_t* o, medata* md, int c) {
    const int W = md->xnb, H = md->ynb;
    int16_t* t = (int16_t*)malloc(sizeof(int16_t) * (size_t)W * H);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) t[(size_t)y * W + x] = block_dc(pic, pw, block_limits(o, pw, ph, x, y));
    int16_t* d = md->dc[c];
    for (int x = 0; x < W; ++x) d[x] = t[x];
    for (int y = 1; y < H - 1; ++y) {
        d[(size_t)y * W] = t[(size_t)y * W];
        for (int x = 1; x < W - 1; ++x) {
#define T(yy, xx) ((int)t[(size_t)(yy) * W + (xx)])
            d[(size_t)y * W + x] = (int16_t)((T(y - 1, x - 1) + 3 * T(y - 1, x) + T(y - 1, x + 1) + 3 * T(y, x - 1) +
                                              3 * T(y, x + 1) + T(y + 1, x - 1) + 3 * T(y + 1, x) + T(y + 1, x + 1) + 8) >>
                                             4);
#undef T
        }
        d[(size_t)y * W + W - 1] = t[(size_t)y * W + W - 1];
    }
    free(t);
}

/* ---------------------------------------------------------------------------------------- */
/* Driver                                                                                    */
/* ---------------------------------------------------------------------------------------- */

int orc_me_depth(int w, int h) {
    return (int)fmin(log((double)w / 12.0) / log(2.0), log((double)h / 12.0) / log(2.0));
}

int orc_motion_estimate(int cformat, int w, int h, const orc_block_params* bp, int nref,
                        const int16_t* const* pic, const int16_t* const* ref1, const int16_t* const* ref2,
                        int luma_depth, float lambda, int stages, int16_t* mv_out, float* cost_out,
                        uint8_t* mode_out, int16_t* dc_out, uint8_t* split_out, float* sbcost_out) {
    if (!bp || nref < 1 || nref > 2 || bp->precision < 1 || bp->precision > 3) return -1;
    olb_t lb[3];
    luma_levels(bp, lb);
    const int xnb = 4 * bp->xnum_sb, ynb = 4 * bp->ynum_sb;
    const int16_t* refs[2] = {ref1[0], nref > 1 ? ref2[0] : ref1[0]};
    int rc = 0;

    /* ---- pel search over the pyramid ---- */
    const int depth = orc_me_depth(w, h);
    if (depth < 0 || depth > 12) return -2;
    int16_t* down[3][13] = {{0}};
    int dw[13], dh[13];
    dw[0] = w;
    dh[0] = h;
    for (int l = 1; l <= depth; ++l) {
        dw[l] = w >> l;
        dh[l] = h >> l;
        dw[l] = w / (1 << l);
        dh[l] = h / (1 << l);
    }
    const int16_t* src0[3] = {pic[0], refs[0], refs[1]};
    for (int s = 0; s < 3; ++s) {
        down[s][0] = (int16_t*)src0[s];
        for (int l = 1; l <= depth; ++l) {
            down[s][l] = (int16_t*)malloc(sizeof(int16_t) * (size_t)dw[l] * dh[l]);
            if (!down[s][l]) return -5;
            if (orc_downconvert(down[s][l - 1], dw[l - 1], dh[l - 1], dw[l - 1], down[s][l], dw[l])) rc = -3;
        }
    }
    medata lev[13];
    int nbx = xnb, nby = ynb;
    if (medata_init(&lev[0], xnb, ynb)) return -5;
    for (int l = 1; l <= depth; ++l) {
        nbx = (nbx >> 1) + (dw[l] % lb[2].xbsep != 0);
        nby = (nby >> 1) + (dh[l] % lb[2].ybsep != 0);
        if (medata_init(&lev[l], nbx, nby)) return -5;
        if (nbx < 2) rc = -4; /* the reference reads outside its vector array below two columns */
    }
    cand_list* L = (cand_list*)malloc(sizeof(cand_list));
    if (rc == 0) {
        for (int l = depth; l >= 0; --l) {
            const medata* guide = (l < depth) ? &lev[l + 1] : &lev[l];
            for (int r = 0; r < nref; ++r)
                match_pic_pel(down[0][l], down[1 + r][l], dw[l], dh[l], &lb[2], &lev[l], guide, r, l, depth, L);
        }
    }
    free(L);
    for (int s = 0; s < 3; ++s)
        for (int l = 1; l <= depth; ++l) free(down[s][l]);
    for (int l = 1; l <= depth; ++l) medata_free(&lev[l]);
    medata* md = &lev[0];

    /* ---- sub-pel refinement ---- */
    int16_t* up[2] = {NULL, NULL};
    if (rc == 0 && stages >= 2) {
        set_lambda_map(md, nref, lambda);
        for (int r = 0; r < nref; ++r) {
            up[r] = (int16_t*)malloc(sizeof(int16_t) * 4 * (size_t)w * h);
            orc_upconvert(refs[r], w, h, w, luma_depth, up[r], 2 * w);
            subpel_pic(pic[0], w, h, up[r], &lb[2], md, r, bp->precision);
        }
    }

    /* ---- mode decision ---- */
    float* sbcost = (float*)calloc((size_t)bp->xnum_sb * bp->ynum_sb, sizeof(float));
    uint8_t* split = (uint8_t*)calloc((size_t)bp->xnum_sb * bp->ynum_sb, 1);
    if (rc == 0 && stages >= 3) {
        mode_ctx M;
        memset(&M, 0, sizeof(M));
        M.pic = pic[0];
        M.pw = w;
        M.ph = h;
        M.up[0] = up[0];
        M.up[1] = up[1] ? up[1] : up[0];
        M.nref = nref;
        M.prec = bp->precision;
        memcpy(M.lb, lb, sizeof(lb));
        M.level_factor[0] = (float)(16 * lb[2].xblen * lb[2].yblen) / (float)(lb[0].xblen * lb[0].yblen);
        M.level_factor[1] = (float)(4 * lb[2].xblen * lb[2].yblen) / (float)(lb[1].xblen * lb[1].yblen);
        M.level_factor[2] = 1.0f;
        medata m0, m1;
        medata_init(&m0, xnb / 4, ynb / 4);
        medata_init(&m1, xnb / 2, ynb / 2);
        M.set[0] = &m0;
        M.set[1] = &m1;
        M.set[2] = md;
        set_lambda_map_level(&m0, 0, md, (float)(1.0 / M.level_factor[0]));
        set_lambda_map_level(&m1, 1, md, (float)(1.0 / M.level_factor[1]));
        M.sbcost = sbcost;
        M.split = split;
        M.xnsb = bp->xnum_sb;
        M.ynsb = bp->ynum_sb;
        for (int ysb = 0; ysb < bp->ynum_sb; ++ysb)
            for (int xsb = 0; xsb < bp->xnum_sb; ++xsb) {
                const size_t sb = (size_t)ysb * bp->xnum_sb + xsb;
                do_level_decn(&M, xsb, ysb, 2);
                float old = sbcost[sb];
                do_level_decn(&M, xsb, ysb, 1);
                if (sbcost[sb] <= old) {
                    old = sbcost[sb];
                    do_level_decn(&M, xsb, ysb, 0);
                }
            }
        medata_free(&m0);
        medata_free(&m1);
        /* SetDC: Y, U, V from the original planes with the component's block parameters */
        for (int c = 0; c < 3; ++c) {
            const int xs = (c && cformat != ORC_444) ? 1 : 0, ys = (c && cformat == ORC_420) ? 1 : 0;
            const olb_t co = make_olb(lb[2].xblen >> xs, lb[2].yblen >> ys, lb[2].xbsep >> xs, lb[2].ybsep >> ys);
            set_dc(pic[c], w >> xs, h >> ys, &co, md, c);
        }
    }

    /* ---- outputs ---- */
    if (rc == 0) {
        const size_t nb = (size_t)xnb * ynb;
        for (int r = 0; r < nref; ++r)
            for (size_t k = 0; k < nb; ++k) {
                mv_out[(r * nb + k) * 2] = (int16_t)md->mv[r][k].x;
                mv_out[(r * nb + k) * 2 + 1] = (int16_t)md->mv[r][k].y;
                cost_out[(r * nb + k) * 3] = md->cost[r][k].SAD;
                cost_out[(r * nb + k) * 3 + 1] = md->cost[r][k].mvcost;
                cost_out[(r * nb + k) * 3 + 2] = md->cost[r][k].total;
            }
        if (stages >= 3) {
            for (size_t k = 0; k < nb; ++k) {
                mode_out[k] = md->mode[k];
                for (int c = 0; c < 3; ++c) dc_out[c * nb + k] = md->dc[c][k];
            }
            for (int k = 0; k < bp->xnum_sb * bp->ynum_sb; ++k) {
                split_out[k] = split[k];
                sbcost_out[k] = sbcost[k];
            }
        }
    }
    free(sbcost);
    free(split);
    free(up[0]);
    free(up[1]);
    medata_free(md);
    return rc;
}
